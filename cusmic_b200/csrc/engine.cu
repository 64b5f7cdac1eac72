// Host side of cusmic_b200: batch layout, workspace pool, launch sequence and
// the C ABI of include/cusmic.h and include/cusmic_b200.h.
//
// One call = init -> prepare -> hole fill -> maxiter x (detect -> grow/update
// -> control -> replace) -> restore, all on the caller's stream, with no host
// synchronisation inside the loop: per-frame activity lives on the device and
// kernels skip frames that stopped (the reference instead copies counts to the
// host after every pass, src/cleaner.cuh:69-76,128-142).  Plans capture the
// same sequence into a CUDA graph whose loop is a device-driven while node.
#include "../../include/cusmic.h"
#include "../../include/cusmic_b200.h"
#include "common.cuh"
#include "detect.cuh"
#include "bulk.cuh"
#include "kernels.cuh"
#include "prepare_bulk.cuh"
#include "prep_detect.cuh"
#include "incremental.cuh"
#include "backward.cuh"
#include "sigmap.cuh"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#ifndef CUSMIC_B200_VERSION
#define CUSMIC_B200_VERSION "0.1.0-b200"
#endif

namespace cb {

struct InvalidArgument : std::invalid_argument {
	using std::invalid_argument::invalid_argument;
};

static void check(cudaError_t e)
{
	if (e == cudaErrorMemoryAllocation)
		throw std::bad_alloc();
	if (e != cudaSuccess)
		throw std::runtime_error(cudaGetErrorString(e));
}

// Injected failures (cusmic_inject_fault): the bounds of the injected device
// waits of calls that start later, and the number of workspace reservations
// still to fail as an exhausted allocator would.
static std::atomic<long long> inject_wait[2] = {{0}, {0}};
static std::atomic<long long> inject_alloc_failures{0};

// True when this reservation is one that an injection makes fail.
static bool injected_alloc_failure()
{
	long long left = inject_alloc_failures.load();
	while (left > 0)
		if (inject_alloc_failures.compare_exchange_weak(left, left - 1))
			return true;
	return false;
}

template <class T> struct DevBuf {
	T *p = nullptr;
	size_t n = 0;
	DevBuf() = default;
	DevBuf(const DevBuf &) = delete;
	DevBuf &operator=(const DevBuf &) = delete;
	void ensure(size_t want)
	{
		const bool fail = injected_alloc_failure();
		if (want <= n && !fail)
			return;
		if (p)
			cudaFree(p);
		p = nullptr;
		n = 0;
		if (want > SIZE_MAX / sizeof(T) || fail)
			throw std::bad_alloc();
		check(cudaMalloc(&p, want * sizeof(T)));
		n = want;
	}
	~DevBuf()
	{
		if (p)
			cudaFree(p);
	}
};

template <class T> struct PinBuf {
	T *p = nullptr;
	size_t n = 0;
	PinBuf() = default;
	PinBuf(const PinBuf &) = delete;
	PinBuf &operator=(const PinBuf &) = delete;
	void ensure(size_t want)
	{
		const bool fail = injected_alloc_failure();
		if (want <= n && !fail)
			return;
		if (p)
			cudaFreeHost(p);
		p = nullptr;
		n = 0;
		if (fail)
			throw std::bad_alloc();
		check(cudaMallocHost(&p, want * sizeof(T)));
		n = want;
	}
	~PinBuf()
	{
		if (p)
			cudaFreeHost(p);
	}
};

// Host threads that copy between the caller's pageable buffers and pinned
// staging memory for the host entry point: a copy is split over the workers
// and the calling thread (one pool per process, shared by concurrent calls).
class CopyPool {
public:
	static CopyPool &get()
	{
		static CopyPool pool;
		return pool;
	}

	// memcpy(dst, src, n), or with src null memset(dst, 0, n), split over the
	// workers and the calling thread.
	void copy(void *dst, const void *src, size_t n)
	{
		const size_t parts = n >= (size_t(2) << 20) ? workers_.size() + 1 : 1;
		const size_t step = ((n + parts - 1) / parts + 63) & ~size_t(63);
		Join join;
		{
			std::lock_guard<std::mutex> g(mu_);
			for (size_t off = step; off < n; off += step) {
				tasks_.push_back(Task{static_cast<char *>(dst) + off,
					src ? static_cast<const char *>(src) + off : nullptr, std::min(step, n - off), &join});
				++join.left;
			}
		}
		cv_.notify_all();
		part(dst, src, std::min(step, n));
		std::unique_lock<std::mutex> lk(join.mu);
		join.cv.wait(lk, [&] { return join.left == 0; });
	}

	// Parts of copies handed to the workers with submit(); wait() returns
	// once all of them are done.  A Join must outlive its parts.
	struct Join {
		std::mutex mu;
		std::condition_variable cv;
		size_t left = 0;
	};

	// The same copy as copy(), split over the workers only, without waiting.
	void submit(Join &join, void *dst, const void *src, size_t n)
	{
		if (workers_.empty() || !n) {
			part(dst, src, n);
			return;
		}
		const size_t parts = workers_.size();
		const size_t step = ((n + parts - 1) / parts + 63) & ~size_t(63);
		{
			std::lock_guard<std::mutex> g(mu_);
			{
				std::lock_guard<std::mutex> j(join.mu);
				join.left += (n + step - 1) / step;
			}
			for (size_t off = 0; off < n; off += step)
				tasks_.push_back(Task{static_cast<char *>(dst) + off,
					src ? static_cast<const char *>(src) + off : nullptr, std::min(step, n - off), &join});
		}
		cv_.notify_all();
	}

	static void wait(Join &join)
	{
		std::unique_lock<std::mutex> lk(join.mu);
		join.cv.wait(lk, [&] { return join.left == 0; });
	}

private:
	static void part(void *dst, const void *src, size_t n)
	{
		if (src)
			std::memcpy(dst, src, n);
		else
			std::memset(dst, 0, n);
	}
	struct Task {
		char *dst;
		const char *src;
		size_t n;
		Join *join;
	};

	CopyPool()
	{
		const unsigned hw = std::thread::hardware_concurrency();
		const unsigned n = hw > 1 ? std::min(hw - 1, 7u) : 0u;
		for (unsigned i = 0; i < n; ++i)
			workers_.emplace_back([this] { run(); });
	}

	~CopyPool()
	{
		{
			std::lock_guard<std::mutex> g(mu_);
			stop_ = true;
		}
		cv_.notify_all();
		for (std::thread &t : workers_)
			t.join();
	}

	void run()
	{
		for (;;) {
			Task t;
			{
				std::unique_lock<std::mutex> lk(mu_);
				cv_.wait(lk, [&] { return stop_ || !tasks_.empty(); });
				if (tasks_.empty())
					return;
				t = tasks_.front();
				tasks_.pop_front();
			}
			part(t.dst, t.src, t.n);
			std::lock_guard<std::mutex> g(t.join->mu);
			if (--t.join->left == 0)
				t.join->cv.notify_all();
		}
	}

	std::mutex mu_;
	std::condition_variable cv_;
	std::deque<Task> tasks_;
	std::vector<std::thread> workers_;
	bool stop_ = false;
};

// Host <-> device copies of the host entry point.  Page-locked caller memory
// is copied by DMA directly.  Pageable memory (which the driver would stage
// itself, one chunk at a time) goes through two pinned slots in chunks: the
// host threads fill (or empty) one slot while the DMA engine moves the other.
struct HostStage {
	static constexpr size_t CHUNK = size_t(16) << 20;
	PinBuf<unsigned char> slot[2];
	cudaEvent_t ev[2] = {nullptr, nullptr};
	bool busy[2] = {false, false}; // a DMA on the slot may still be in flight
	int next = 0;

	~HostStage()
	{
		for (cudaEvent_t e : ev)
			if (e)
				cudaEventDestroy(e);
	}

	static bool pinned(const void *p)
	{
		cudaPointerAttributes a;
		if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
			cudaGetLastError();
			return false;
		}
		return a.type == cudaMemoryTypeHost;
	}

	// A free slot: its last DMA has completed.
	int take()
	{
		const int k = next;
		next ^= 1;
		if (!ev[k])
			check(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
		slot[k].ensure(CHUNK);
		if (busy[k])
			check(cudaEventSynchronize(ev[k]));
		busy[k] = false;
		return k;
	}

	void in(void *dst, const void *src, size_t n, cudaStream_t s)
	{
		if (!n)
			return;
		if (pinned(src)) {
			check(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s));
			return;
		}
		for (size_t off = 0; off < n; off += CHUNK) {
			const size_t len = std::min(CHUNK, n - off);
			const int k = take();
			CopyPool::get().copy(slot[k].p, static_cast<const char *>(src) + off, len);
			check(cudaMemcpyAsync(static_cast<char *>(dst) + off, slot[k].p, len, cudaMemcpyHostToDevice, s));
			check(cudaEventRecord(ev[k], s));
			busy[k] = true;
		}
	}

	// Returns with the copy complete.
	void out(void *dst, const void *src, size_t n, cudaStream_t s)
	{
		if (!n)
			return;
		if (pinned(dst)) {
			check(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s));
			check(cudaStreamSynchronize(s));
			return;
		}
		const size_t nch = (n + CHUNK - 1) / CHUNK;
		int k[2] = {-1, -1};
		auto issue = [&](size_t i) {
			const size_t off = i * CHUNK, len = std::min(CHUNK, n - off);
			k[i & 1] = take();
			check(cudaMemcpyAsync(slot[k[i & 1]].p, static_cast<const char *>(src) + off, len,
				cudaMemcpyDeviceToHost, s));
			check(cudaEventRecord(ev[k[i & 1]], s));
			busy[k[i & 1]] = true;
		};
		issue(0);
		for (size_t i = 0; i < nch; ++i) {
			if (i + 1 < nch)
				issue(i + 1);
			const int ki = k[i & 1];
			check(cudaEventSynchronize(ev[ki]));
			busy[ki] = false;
			const size_t off = i * CHUNK;
			CopyPool::get().copy(static_cast<char *>(dst) + off, slot[ki].p, std::min(CHUNK, n - off));
		}
	}
};

// Launch parameters (include/cusmic_b200.h, struct cusmic_tuning).
static std::mutex tuning_mu;
static std::vector<cusmic_tuning> tuning_table;

static cusmic_tuning default_tuning(size_t)
{
	return cusmic_tuning{SIZE_MAX, 0, BK_BLOCKS_PER_SM, 8, 8};
}

static cusmic_tuning tuning_for(size_t total_px)
{
	std::lock_guard<std::mutex> lock(tuning_mu);
	for (const cusmic_tuning &t : tuning_table)
		if (total_px <= t.max_pixels)
			return t;
	return default_tuning(total_px);
}

// Host description of one batch.
struct Layout {
	std::vector<FrameDesc> frames;
	std::vector<long long> bit_off; // word offset of each frame within a plane
	std::vector<long long> row_off; // first row of each frame in the row marks
	long long row_words = 0;        // row marks of all frames, padded to 4
	std::vector<int4> bulk;   // sig_bulk_kernel items {frame, x0, y0, first threshold of the frame}
	std::vector<int4> grow;   // grow_kernel items {frame, y0, first word, y1}
	std::vector<FloorJob> jobs; // floor blocks of each distinct error map and noise-model frame
	std::vector<long long> thr_base; // per frame: first floor of its blocks
	long long nthr = 0;
	std::vector<int2> rows;
	std::vector<long long> offsets; // first output pixel of each frame
	long long total_words = 0;  // all planes
	long long plane_words = 0;  // one plane of every frame
	size_t total_px = 0;
	DetectParams prm{};
	int maxiter = 0;
	int error_frames = 0; // frames with an error map (a rebound plan keeps which)
	// Kernel choices that depend on the buffers' alignment (a rebound plan
	// whose choices change is captured again): the bulk-staged prepare, and
	// prepare with the dense detection in one kernel (prep_detect_kernel).
	bool prep_bulk = false, fused = false;
	cusmic_tuning tune{};
	long long poison_wait[2] = {0, 0}; // injected failures in force when the batch was laid out
};

struct DeviceInfo {
	int sms = 0;
};

static DeviceInfo device_info(int dev)
{
	static std::mutex mu;
	static std::vector<DeviceInfo> cache;
	std::lock_guard<std::mutex> lock(mu);
	if ((int)cache.size() <= dev)
		cache.resize(dev + 1);
	DeviceInfo &d = cache[dev];
	if (!d.sms) { // first use on this (the current) device
		check(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
		for (const void *k : {(const void *)prepare_bulk_kernel<false, false>,
			     (const void *)prepare_bulk_kernel<true, false>,
			     (const void *)prepare_bulk_kernel<false, true>,
			     (const void *)prepare_bulk_kernel<true, true>})
			check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB_SMEM));
	}
	return d;
}

struct Workspace {
	int device = -1;
	DevBuf<FrameDesc> frames;
	DevBuf<FrameState> state;
	DevBuf<int2> rows;
	DevBuf<uint32_t> bits;
	DevBuf<uint32_t> rowmarks; // growth row marks, then CHG row marks (row_words each)
	DevBuf<uint2> targets;
	DevBuf<uint8_t> radius; // per target: window radius of its last replacement
	DevBuf<int2> dirty;     // dirty-row list of an incremental pass
	DevBuf<unsigned> sel;   // targets the replacement after a pass visits
	DevBuf<Seed> seeds;     // seed slots of the noise-model candidates
	DevBuf<double> work;    // working pixels of the frames with a background
	DevBuf<double> sigmap;  // first-pass sig_raw, then noise, of noise-model frames (2 x pixels)
	DevBuf<uint2> cands;
	DevBuf<int4> bulk;
	DevBuf<int4> grow;
	DevBuf<FloorJob> jobs;
	DevBuf<BlockFloor> floors;
	DevBuf<PreCand> pre;
	DevBuf<int> pre_counts;
	DevBuf<Control> ctl;
	DevBuf<long long> offsets;
	PinBuf<unsigned char> stage;
	PinBuf<FrameState> hstate;
	// Host-API staging of inputs and outputs.
	DevBuf<double> hdata, herror, hgain, hrn, hbg, hclean;
	DevBuf<uint8_t> hmask, hout;
	HostStage stage_io; // pageable host buffers of the host entry point
	DevBuf<unsigned> hflags; // failed map checks of the host entry point
	// Host-buffer batch (cusmic_batch_host): maps shared by several frames,
	// and the pinned copies of a chunk's state and map-check flags.
	DevBuf<double> hshared;
	DevBuf<uint8_t> hshared_mask;
	PinBuf<unsigned> hflags_host;
	// Its sparse return: the cleaned values along the target list, the
	// list's length, and pinned host copies of list and values.
	DevBuf<double> hsp_val;
	PinBuf<unsigned long long> hcount;
	PinBuf<uint2> hsp_idx_host;
	PinBuf<double> hsp_val_host;
};

static std::mutex pool_mu;
static std::vector<std::unique_ptr<Workspace>> pool;

struct Lease {
	std::unique_ptr<Workspace> ws;
	explicit Lease(int dev)
	{
		std::lock_guard<std::mutex> lock(pool_mu);
		for (auto it = pool.begin(); it != pool.end(); ++it)
			if ((*it)->device == dev) {
				ws = std::move(*it);
				pool.erase(it);
				break;
			}
		if (!ws) {
			ws.reset(new Workspace);
			ws->device = dev;
		}
	}
	~Lease()
	{
		if (!ws)
			return;
		std::lock_guard<std::mutex> lock(pool_mu);
		pool.push_back(std::move(ws));
	}
	Workspace *operator->() { return ws.get(); }
	Workspace &operator*() { return *ws; }
};

// Options and scalars of frame f after per-frame overrides.
struct FrameScalars {
	double gain, rn, bg;
};

static FrameScalars scalars_for(const cusmic_options &o, const cusmic_frame_scalars *sc, size_t f)
{
	FrameScalars r{o.gain, o.readnoise, o.background};
	if (sc) {
		if (!std::isnan(sc[f].gain))
			r.gain = sc[f].gain;
		if (!std::isnan(sc[f].readnoise))
			r.rn = sc[f].readnoise;
		r.bg = sc[f].background;
	}
	return r;
}

// Reference src/api.cu:47-81, generalised to ragged shapes and per-frame
// scalars.  Messages match the reference's.
static void check_arguments(const cusmic_image *ims, size_t nf, const cusmic_options *o,
	const cusmic_frame_scalars *sc, const void *clean, const void *mask, bool same_shape)
{
	if (!ims || !o || !clean || !mask || !nf || nf > 65535)
		throw InvalidArgument("invalid images, batch size or output buffers");
	const size_t w0 = ims[0].width, h0 = ims[0].height;
	size_t total = 0;
	for (size_t f = 0; f < (same_shape ? 1 : nf); ++f) {
		size_t w = ims[f].width, h = ims[f].height;
		if (!w || !h || w > size_t(INT_MAX) / 4 / h)
			throw InvalidArgument("invalid image dimensions");
		size_t n = w * h;
		if ((same_shape && nf > SIZE_MAX / sizeof(double) / n) ||
			total > SIZE_MAX / sizeof(double) - n)
			throw InvalidArgument("batch is too large");
		total += n;
	}
	if (o->maxiter < 0 || o->border < 0 || o->border > CUSMIC_WRAP || !std::isfinite(o->contrast) ||
		o->contrast < 0 || !std::isfinite(o->cr_threshold) || o->cr_threshold < 0 ||
		!std::isfinite(o->neighbor_threshold) || o->neighbor_threshold < 0)
		throw InvalidArgument("invalid detection settings");
	for (size_t f = 0; f < nf; ++f) {
		const cusmic_image &im = ims[f];
		if (!im.data || (same_shape && (im.width != w0 || im.height != h0)))
			throw InvalidArgument("frames must have data and the same shape");
		FrameScalars s = scalars_for(*o, sc, f);
		if (!im.error) {
			bool needs_gain = o->maxiter || !std::isnan(s.gain);
			if (!im.gain && needs_gain && (!std::isfinite(s.gain) || s.gain <= 0))
				throw InvalidArgument("positive gain or error is required");
			if (!im.readnoise && (!std::isfinite(s.rn) || s.rn < 0))
				throw InvalidArgument("read noise must be finite and nonnegative");
		}
		if (!im.background && !std::isnan(s.bg) && !std::isfinite(s.bg))
			throw InvalidArgument("background must be finite");
	}
}

// Device buffers hold float64 values: every pointer must be 8-byte aligned.
static void check_device_alignment(const cusmic_image *ims, size_t nf, const double *clean)
{
	auto bad = [](const void *p) { return ((uintptr_t)p & 7) != 0; };
	bool any = bad(clean);
	for (size_t f = 0; f < nf; ++f)
		any = any || bad(ims[f].data) || bad(ims[f].error) || bad(ims[f].gain) ||
			bad(ims[f].readnoise) || bad(ims[f].background);
	if (any)
		throw InvalidArgument("float64 buffers must be 8-byte aligned");
}

// Rows per item of the dense detection kernel: 32, or fewer (16, 8, 4) while
// the batch has fewer items than the kernel has resident blocks, so small
// frames still spread over the GPU.
static int item_rows(const cusmic_image *ims, size_t nf, int target_items)
{
	int rows = BK_ROWS;
	while (rows > 4) {
		long long items = 0;
		for (size_t f = 0; f < nf; ++f)
			items += (long long)((ims[f].width + BK_COLS - 1) / BK_COLS) *
				(long long)((ims[f].height + rows - 1) / rows);
		if (items >= target_items)
			break;
		rows /= 2;
	}
	return rows;
}

// The prepare kernels that suit every frame of a batch (see Layout).
static void choose_kernels(Layout &L)
{
	L.prep_bulk = true;
	L.fused = L.maxiter > 0;
	for (const FrameDesc &fd : L.frames) {
		L.prep_bulk = L.prep_bulk && prep_bulk_ok(fd);
		L.fused = L.fused && prep_detect_ok(fd);
	}
}

static Layout make_layout(const cusmic_image *ims, size_t nf, const cusmic_options &o,
	const cusmic_frame_scalars *sc, double *clean, uint8_t *mask, const DeviceInfo &di)
{
	size_t all_px = 0;
	for (size_t f = 0; f < nf; ++f)
		all_px += ims[f].width * ims[f].height;
	const cusmic_tuning tune = tuning_for(all_px);
	const int rows_per_item = tune.dense_rows ? tune.dense_rows
		: item_rows(ims, nf, di.sms * tune.dense_blocks_per_sm);
	Layout L;
	L.tune = tune;
	L.poison_wait[0] = inject_wait[0].load();
	L.poison_wait[1] = inject_wait[1].load();
	L.maxiter = o.maxiter;
	L.prm.contrast = o.contrast;
	L.prm.cr = o.cr_threshold;
	L.prm.nb = o.neighbor_threshold;
	L.prm.tmin = std::fmin(o.cr_threshold, o.neighbor_threshold);
	L.prm.thi2 = 2 * o.cr_threshold * (1 - 1e-12);
	L.prm.tlo2 = 2 * o.neighbor_threshold * (1 - 1e-12);
	L.prm.mode = o.border;
	L.frames.resize(nf);
	L.bit_off.resize(nf);
	L.thr_base.assign(nf, -1);
	std::map<const double *, std::vector<std::pair<int, long long>>> maps; // error map -> {frame, base}
	size_t px = 0;
	long long words = 0;
	for (size_t f = 0; f < nf; ++f) {
		const cusmic_image &im = ims[f];
		FrameDesc &d = L.frames[f];
		FrameScalars s = scalars_for(o, sc, f);
		d.data = im.data;
		d.error = im.error;
		L.error_frames += im.error != nullptr;
		d.gain_map = im.error ? nullptr : im.gain;
		d.rn_map = im.error ? nullptr : im.readnoise;
		d.bg_map = im.background;
		d.mask = im.mask;
		d.clean = clean + px;
		d.mask_out = mask + px;
		d.gain = s.gain;
		d.rn = s.rn;
		d.bg = s.bg;
		d.w = (int)im.width;
		d.h = (int)im.height;
		d.words = (d.w + 31) / 32;
		d.plane = (long long)d.h * d.words;
		d.has_bg = im.background != nullptr || !std::isnan(s.bg);
		d.bits = nullptr;
		L.bit_off[f] = words;
		L.row_off.push_back(L.row_words);
		L.row_words += d.h;
		L.offsets.push_back((long long)px);
		words += d.plane;
		px += (size_t)d.w * d.h;
		for (int y = 0; y < d.h; ++y)
			L.rows.push_back(make_int2((int)f, y));
		// Thresholds: frames of the same shape that share an error map share
		// them; every noise-model frame has its own.
		const int bw = (d.w + FLOOR_BLOCK - 1) / FLOOR_BLOCK, bh = (d.h + FLOOR_BLOCK - 1) / FLOOR_BLOCK;
		long long base = -1;
		if (d.error)
			for (const auto &m : maps[d.error])
				if (L.frames[m.first].w == d.w && L.frames[m.first].h == d.h)
					base = m.second;
		if (base < 0) {
			base = L.nthr;
			if (d.error)
				maps[d.error].push_back({(int)f, base});
			for (int by = 0; by < bh; ++by)
				for (int bx = 0; bx < bw; ++bx)
					L.jobs.push_back(FloorJob{(int)f, bx * FLOOR_BLOCK, by * FLOOR_BLOCK,
						d.error ? 0 : 1, base + (long long)by * bw + bx});
			L.nthr += (long long)bw * bh;
		}
		L.thr_base[f] = base;
		for (int ty = 0; ty < d.h; ty += rows_per_item)
			for (int tx = 0; tx < d.w; tx += BK_COLS)
				L.bulk.push_back(make_int4((int)f, tx, ty, std::min(ty + rows_per_item, d.h)));
		for (int ty = 0; ty < d.h; ty += GROW_ROWS)
			for (int k0 = 0; k0 < d.words; k0 += 32)
				L.grow.push_back(make_int4((int)f, ty, k0, std::min(ty + GROW_ROWS, d.h)));
	}
	L.total_px = px;
	choose_kernels(L);
	L.row_words = (L.row_words + 3) & ~3ll;
	// Planes padded to 4 words, so every plane starts on a 16-byte boundary.
	L.plane_words = (words + 3) & ~3ll;
	L.total_words = (long long)N_PLANES * L.plane_words;
	for (FrameDesc &d : L.frames)
		d.pstride = L.plane_words;
	return L;
}

static int grid_for_rows(const DeviceInfo &di, size_t nrows, int blocks_per_sm = 8)
{
	size_t blocks = (nrows + 7) / 8;
	size_t cap = (size_t)di.sms * blocks_per_sm;
	return (int)(blocks < 1 ? 1 : blocks > cap ? cap : blocks);
}

// The device address of page-locked host memory (mapped into the device's
// address space).
static const void *host_device_ptr(const void *p)
{
	void *d = nullptr;
	check(cudaHostGetDevicePointer(&d, const_cast<void *>(p), 0));
	return d;
}

// Allocate the workspace for L and upload descriptors (stream-ordered).
// `mapped`: a kernel reads them from the page-locked staging buffer, so the
// upload does not queue behind large copies on the copy engine (the host
// batch entry point keeps its inbound copies running while it cleans).
static void upload(Workspace &ws, Layout &L, cudaStream_t s, bool mapped = false)
{
	const size_t nf = L.frames.size();
	ws.frames.ensure(nf);
	ws.state.ensure(nf);
	ws.bulk.ensure(L.bulk.size() ? L.bulk.size() : 1);
	ws.grow.ensure(L.grow.size() ? L.grow.size() : 1);
	ws.jobs.ensure(L.jobs.size() ? L.jobs.size() : 1);
	ws.floors.ensure(L.nthr ? (size_t)L.nthr : 1);
	ws.rows.ensure(L.rows.size());
	ws.ctl.ensure(1);
	ws.offsets.ensure(nf);
	if (L.maxiter) {
		ws.bits.ensure((size_t)L.total_words);
		ws.rowmarks.ensure(2 * (size_t)L.row_words);
		ws.targets.ensure(L.total_px);
		ws.radius.ensure(L.total_px);
		ws.dirty.ensure(L.rows.size());
		ws.sel.ensure(L.total_px);
		if (L.error_frames < (int)nf)
			ws.seeds.ensure(L.total_px);
		ws.cands.ensure(L.total_px);
		ws.pre.ensure(L.bulk.size() * BK_CWARPS * (size_t)BK_REGION);
		ws.pre_counts.ensure(L.bulk.size() * BK_CWARPS);
	}
	// A frame with a background keeps its working pixels (data + background)
	// in the workspace, and prepare writes its output pixels at once (the
	// reference's (x + bg) - bg), so restore writes only the flagged ones
	// instead of reading and rewriting the whole frame.
	bool any_bg = false;
	for (const FrameDesc &d : L.frames)
		any_bg = any_bg || d.has_bg;
	if (L.maxiter && any_bg)
		ws.work.ensure(L.total_px);
	if (L.maxiter && L.error_frames < (int)nf)
		ws.sigmap.ensure(2 * L.total_px);
	for (size_t f = 0; f < nf; ++f) {
		L.frames[f].bits = L.maxiter ? ws.bits.p + L.bit_off[f] : nullptr;
		L.frames[f].floors = L.maxiter ? ws.floors.p + L.thr_base[f] : nullptr;
		L.frames[f].rowcand = L.maxiter ? ws.rowmarks.p + L.row_off[f] : nullptr;
		L.frames[f].rowchg = L.maxiter ? ws.rowmarks.p + L.row_words + L.row_off[f] : nullptr;
		L.frames[f].out = L.frames[f].clean;
		const bool sm = L.maxiter && !L.frames[f].error;
		L.frames[f].sig_raw = sm ? ws.sigmap.p + L.offsets[f] : nullptr;
		L.frames[f].noise = sm ? ws.sigmap.p + L.total_px + L.offsets[f] : nullptr;
		if (L.maxiter && L.frames[f].has_bg)
			L.frames[f].clean = ws.work.p + L.offsets[f];
	}
	// Every descriptor array goes through one pinned staging buffer.  The
	// previous call using this workspace synchronised before returning, so
	// the buffer is free.
	struct Part {
		void *dst;
		const void *src;
		size_t bytes;
	};
	const Part parts[] = {
		{ws.frames.p, L.frames.data(), nf * sizeof(FrameDesc)},
		{ws.rows.p, L.rows.data(), L.rows.size() * sizeof(int2)},
		{ws.bulk.p, L.bulk.data(), L.bulk.size() * sizeof(int4)},
		{ws.grow.p, L.grow.data(), L.grow.size() * sizeof(int4)},
		{ws.jobs.p, L.jobs.data(), L.jobs.size() * sizeof(FloorJob)},
		{ws.offsets.p, L.offsets.data(), nf * sizeof(long long)},
	};
	size_t total = 0;
	for (const Part &q : parts)
		total += (q.bytes + 15) & ~size_t(15);
	ws.stage.ensure(total);
	WordCopies wc{};
	const unsigned char *dstage = mapped
		? static_cast<const unsigned char *>(host_device_ptr(ws.stage.p)) : nullptr;
	size_t at = 0;
	for (const Part &q : parts) {
		if (q.bytes) {
			std::memcpy(ws.stage.p + at, q.src, q.bytes);
			if (mapped) {
				static_assert(sizeof(FrameDesc) % 8 == 0 && sizeof(FloorJob) % 8 == 0, "8-byte parts");
				wc.part[wc.n++] = WordCopy{reinterpret_cast<const unsigned long long *>(dstage + at),
					static_cast<unsigned long long *>(q.dst), (long long)(q.bytes / 8)};
			} else {
				check(cudaMemcpyAsync(q.dst, ws.stage.p + at, q.bytes, cudaMemcpyHostToDevice, s));
			}
		}
		at += (q.bytes + 15) & ~size_t(15);
	}
	if (mapped && wc.n)
		word_copy_kernel<<<32, 256, 0, s>>>(wc);
}

struct GraphLoop {
	cudaGraphConditionalHandle handle = 0;
	bool use = false;
};

// Kernel kinds reported by cusmic_plan_profile().
enum KernelKind { K_INIT, K_PREPARE, K_FILL, K_SIGRAW, K_CAND, K_SEED, K_GROW, K_CONTROL,
	K_REPLACE, K_RESTORE, K_COPY, K_LOW, K_CLASSIFY, K_FLOOR, K_RECLASS, K_DIRTY, K_SIGMAP, K_KINDS };

// Optional CUDA-event timer: an event after every launch on the launching
// stream, so each kernel's duration is the gap to the previous event.
struct Recorder {
	std::vector<cudaEvent_t> events;
	std::vector<int> kinds;
	cudaStream_t s = nullptr;
	void begin(cudaStream_t stream)
	{
		s = stream;
		mark(-1);
	}
	void mark(int kind)
	{
		cudaEvent_t e;
		check(cudaEventCreate(&e));
		check(cudaEventRecord(e, s));
		events.push_back(e);
		kinds.push_back(kind);
	}
	~Recorder()
	{
		for (cudaEvent_t e : events)
			cudaEventDestroy(e);
	}
};

static inline void mark(Recorder *r, int kind)
{
	if (r)
		r->mark(kind);
}

// Grids of the kernels with a thread per work item (grid-stride loops): the
// blocks that fit an SM at their register use (80 per thread for the
// first-window kernels, 120 for candidate_map_kernel), so a short list costs
// no waves of idle blocks.
constexpr int WINDOW_BLOCKS_PER_SM = 3, MAP_BLOCKS_PER_SM = 2;

// One detection pass.  The first pass of a call is full: the dense kernel
// lists every candidate and the classification fills the HIGH / LOW planes.
// Later passes are incremental (incremental.cuh): they start from the pixels
// that the last replacement changed and keep the other bits.
static void launch_pass(Workspace &ws, const Layout &L, const DeviceInfo &di, cudaStream_t s,
	const GraphLoop &gl, bool incremental, Recorder *rec = nullptr)
{
	const int nf = (int)L.frames.size(), nrows = (int)L.rows.size();
	const int nbulk = (int)L.bulk.size();
	const int cap = di.sms * L.tune.dense_blocks_per_sm, sparse = di.sms * L.tune.sparse_blocks_per_sm;
	const int rowb = L.tune.row_blocks_per_sm;
	if (incremental) {
		// The dirty-row scan also zeroes FRESH of every frame (its growth
		// visits a row list); the full pass finds S1, S2, CAND, FRESH and the
		// growth row marks zeroed by the prologue.
		const long long n16 = L.plane_words / 4; // 16-byte words of one plane
		const long long need = ((n16 > nrows ? n16 : nrows) + 255) / 256;
		const int tb = (int)(need < di.sms * 4 ? need : di.sms * 4);
		dirty_rows_kernel<<<tb, 256, 0, s>>>(ws.frames.p, ws.state.p, ws.rows.p, nrows, L.prm.mode,
			ws.ctl.p, ws.dirty.p, reinterpret_cast<uint4 *>(ws.bits.p + P_FRESH * L.plane_words), n16);
		mark(rec, K_DIRTY);
		const int rgrid = grid_for_rows(di, nrows, rowb);
		if (L.error_frames)
			incremental_rows_kernel<false><<<rgrid, 256, 0, s>>>(ws.frames.p, ws.dirty.p,
				&ws.ctl.p->n_dirty, L.prm, ws.ctl.p, ws.cands.p);
		if (L.error_frames < nf)
			incremental_rows_kernel<true><<<rgrid, 256, 0, s>>>(ws.frames.p, ws.dirty.p,
				&ws.ctl.p->n_dirty, L.prm, ws.ctl.p, ws.cands.p);
		mark(rec, K_RECLASS);
	} else {
		// (A fused batch's prologue listed the pixels already.)
		if (!L.fused) {
			sig_bulk_kernel<<<nbulk < cap ? nbulk : cap, BK_THREADS, 0, s>>>(ws.frames.p, ws.state.p,
				ws.bulk.p, nbulk, L.prm, ws.ctl.p, ws.pre.p, ws.pre_counts.p);
			mark(rec, K_SIGRAW);
		}
		const int cgrid = (nbulk * BK_CWARPS + 7) / 8 < sparse ? (nbulk * BK_CWARPS + 7) / 8 : sparse;
		classify_kernel<<<cgrid, 256, 0, s>>>(ws.frames.p, ws.state.p, ws.bulk.p, nbulk, ws.pre.p,
			ws.pre_counts.p, L.prm, ws.ctl.p, ws.cands.p);
		mark(rec, K_CLASSIFY);
		if (L.error_frames < nf) { // the noise-model candidates' sig_raw map
			const int ng = (int)L.grow.size(), need = (ng + 7) / 8, gcap = di.sms * 8;
			region_list_kernel<<<need < gcap ? need : gcap, 256, 0, s>>>(ws.frames.p, ws.state.p, ws.grow.p,
				ng, ws.ctl.p, ws.targets.p);
			region_sig_kernel<<<di.sms * 8, 256, 0, s>>>(ws.frames.p, ws.targets.p, ws.ctl.p, L.prm);
			mark(rec, K_SIGMAP);
		}
	}
	// One launch per kind of frame in the batch: each variant compiles only
	// its noise path (error map or noise model).  Error-map seeds are tested
	// by the candidate's own warp; noise-model seeds by seed_kernel.
	const bool model = L.error_frames < nf;
	if (L.error_frames)
		candidate_seed_kernel<PATH_ERROR><<<sparse, 256, 0, s>>>(ws.frames.p, ws.cands.p, L.prm,
			ws.ctl.p, model ? ws.seeds.p : nullptr, !incremental);
	if (model && incremental)
		candidate_high_kernel<PATH_MODEL><<<sparse, 256, 0, s>>>(ws.frames.p, ws.cands.p, L.prm,
			ws.ctl.p, ws.seeds.p, 0);
	else if (model) // the first pass: windows from the sig_raw map, a thread per candidate
		candidate_map_kernel<<<di.sms * MAP_BLOCKS_PER_SM, 256, 0, s>>>(ws.frames.p, ws.cands.p, L.prm,
			ws.ctl.p, ws.seeds.p);
	mark(rec, K_CAND);
	if (model) {
		seed_kernel<<<sparse, 256, 0, s>>>(ws.frames.p, ws.seeds.p, L.prm, ws.ctl.p, !incremental);
		mark(rec, K_SEED);
	}
	if (L.error_frames)
		candidate_low_kernel<PATH_ERROR><<<sparse, 256, 0, s>>>(ws.frames.p, ws.cands.p, L.prm,
			ws.ctl.p, !incremental);
	if (L.error_frames < nf)
		candidate_low_kernel<PATH_MODEL><<<sparse, 256, 0, s>>>(ws.frames.p, ws.cands.p, L.prm,
			ws.ctl.p, !incremental);
	mark(rec, K_LOW);
	// Growth visits the items holding marked rows.
	{
		const int ng = (int)L.grow.size(), need = (ng + 7) / 8, gcap = di.sms * rowb;
		grow_kernel<<<need < gcap ? need : gcap, 256, 0, s>>>(ws.frames.p, ws.state.p, ws.grow.p, ng,
			ws.targets.p, ws.ctl.p);
	}
	mark(rec, K_GROW);
	control_kernel<<<1, 1024, 0, s>>>(ws.state.p, nf, ws.ctl.p, gl.handle, gl.use ? 1 : 0);
	mark(rec, K_CONTROL);
	const int tb = di.sms * 4;
	replace_select_kernel<<<tb, 256, 0, s>>>(ws.frames.p, ws.state.p, ws.targets.p,
		&ws.ctl.p->n_targets, ws.radius.p, ws.ctl.p, ws.sel.p,
		reinterpret_cast<uint4 *>(ws.rowmarks.p + L.row_words), L.row_words / 4);
	replace_kernel<<<di.sms * WINDOW_BLOCKS_PER_SM, 256, 0, s>>>(ws.frames.p, ws.state.p, ws.targets.p,
		&ws.ctl.p->n_targets, ws.sel.p, &ws.ctl.p->n_sel, ws.radius.p);
	mark(rec, K_REPLACE);
}

// prepare: the bulk-staged kernel when every frame suits it; else one
// compiled for noise-model frames without maps, with twice the unroll, when
// every frame is of that kind; otherwise the kernel that decides per row
// (faster for error-map frames than any specialisation that was timed).
static void launch_prepare(Workspace &ws, const Layout &L, const DeviceInfo &di, cudaStream_t s)
{
	bool model = true, rowmin = false, out = false;
	const bool bulk = L.prep_bulk;
	for (const FrameDesc &fd : L.frames) {
		const int kind = prep_kind(fd);
		model = model && kind == PREP_MODEL;
		rowmin = rowmin || kind == PREP_MODEL || kind == PREP_MODEL_MAPS;
		out = out || (fd.out && fd.out != fd.clean);
	}
	const int nrows = (int)L.rows.size();
	// Each variant is compiled for what the batch has (row minima, separate
	// outputs): the kernels are issue-bound, and an unused branch costs.
	if (bulk) {
		const int need = (nrows + PB_WARPS - 1) / PB_WARPS, cap = di.sms * PB_BLOCKS;
		const int grid = need < cap ? need : cap;
		auto k = rowmin ? (out ? prepare_bulk_kernel<true, true> : prepare_bulk_kernel<true, false>)
				: (out ? prepare_bulk_kernel<false, true> : prepare_bulk_kernel<false, false>);
		k<<<grid, 32 * PB_WARPS, PB_SMEM, s>>>(ws.frames.p, ws.state.p, ws.rows.p, nrows, ws.ctl.p,
			ws.cands.p);
		return;
	}
	const int grid = grid_for_rows(di, nrows, L.tune.row_blocks_per_sm);
	auto k = model ? (out ? prepare_kernel<PREP_MODEL, 2 * ROW_UNROLL, true>
			       : prepare_kernel<PREP_MODEL, 2 * ROW_UNROLL, false>)
		       : (out ? prepare_kernel<PREP_ANY, ROW_UNROLL, true> : prepare_kernel<PREP_ANY, ROW_UNROLL, false>);
	k<<<grid, 256, 0, s>>>(ws.frames.p, ws.state.p, ws.rows.p, nrows, ws.ctl.p, ws.cands.p);
}

static void launch_prologue(Workspace &ws, const Layout &L, const DeviceInfo &di, cudaStream_t s,
	Recorder *rec = nullptr)
{
	const int nf = (int)L.frames.size(), nrows = (int)L.rows.size();
	if (!L.maxiter) {
		init_kernel<<<(nf + 255) / 256, 256, 0, s>>>(ws.state.p, nf, ws.ctl.p, L.maxiter,
			(unsigned long long)L.total_px, L.poison_wait[0], L.poison_wait[1]);
		mark(rec, K_INIT);
		copy_kernel<<<grid_for_rows(di, nrows), 256, 0, s>>>(ws.frames.p, ws.rows.p, nrows);
		mark(rec, K_COPY);
		return;
	}
	// The same launch zeroes the bit planes from CRMASK to CHG and both
	// row-mark arrays: nothing else writes them before the first pass, which
	// therefore clears nothing itself.  prepare writes every word of HOLE,
	// EXCL and DONOR, and of ROWMIN on noise-model frames (the only frames
	// whose ROWMIN is read).  Planes and row marks are padded to 16 bytes.
	static_assert(P_HOLE == 0 && P_EXCL == 1 && P_DONOR == 2 && P_CRMASK == 3 &&
		P_ROWMIN == N_PLANES - 1, "plane order");
	const long long z16 = (long long)(P_ROWMIN - P_CRMASK) * L.plane_words / 4;
	const long long r16 = 2 * L.row_words / 4;
	const long long zb = (std::max(z16, r16) + 255) / 256, fb = (nf + 255) / 256,
		zcap = (long long)di.sms * 8;
	uint4 *const zero = reinterpret_cast<uint4 *>(ws.bits.p + P_CRMASK * L.plane_words);
	uint4 *const zero2 = reinterpret_cast<uint4 *>(ws.rowmarks.p);
	if (L.fused) {
		// The error-map floors (they read the maps only) in the same launch
		// as the state and the zeroing, then prepare with the first pass's
		// dense detection in one kernel, then the hole fill.
		const long long jb = ((long long)L.jobs.size() + 7) / 8;
		prep_init_kernel<<<(int)std::max({fb, std::min(zb, zcap), std::min(jb, zcap)}), 256, 0, s>>>(
			ws.state.p, nf, ws.ctl.p, L.maxiter, (unsigned long long)L.total_px, L.poison_wait[0],
			L.poison_wait[1], zero, z16, zero2, r16, ws.frames.p, ws.jobs.p, (int)L.jobs.size(), L.prm,
			ws.floors.p);
		mark(rec, K_INIT); // the state, the zeroed planes and the floors
		const int nbulk = (int)L.bulk.size(), pcap = di.sms * PD_BLOCKS_PER_SM;
		prep_detect_kernel<<<nbulk < pcap ? nbulk : pcap, BK_THREADS, 0, s>>>(ws.frames.p, ws.state.p,
			ws.bulk.p, nbulk, L.prm, ws.ctl.p, ws.cands.p, ws.pre.p, ws.pre_counts.p);
		mark(rec, K_PREPARE);
		fill_list_kernel<<<di.sms * WINDOW_BLOCKS_PER_SM, 256, 0, s>>>(ws.frames.p, ws.state.p,
			ws.cands.p, &ws.ctl.p->n_holes);
		mark(rec, K_FILL);
		return;
	}
	init_kernel<<<(int)std::max(fb, std::min(zb, zcap)), 256, 0, s>>>(ws.state.p, nf, ws.ctl.p,
		L.maxiter, (unsigned long long)L.total_px, L.poison_wait[0], L.poison_wait[1], zero, z16, zero2,
		r16);
	mark(rec, K_INIT); // the state and the zeroed planes
	launch_prepare(ws, L, di, s);
	mark(rec, K_PREPARE);
	// Block floors: error-map thresholds; noise-model keys from prepare's row
	// minima of the non-hole pixels, which the hole fill and every later
	// replacement lower with the values they write.
	if (!L.jobs.empty()) {
		const int nj = (int)L.jobs.size(), cap = di.sms * 8;
		floor_kernel<<<(nj + 7) / 8 < cap ? (nj + 7) / 8 : cap, 256, 0, s>>>(ws.frames.p, ws.jobs.p,
			nj, L.prm, ws.floors.p);
		if (L.error_frames < nf)
			model_floor_kernel<<<(nj + 255) / 256 < cap ? (nj + 255) / 256 : cap, 256, 0, s>>>(
				ws.frames.p, ws.jobs.p, nj, ws.floors.p);
		mark(rec, K_FLOOR);
	}
	// The hole list lives in the candidate buffer until the first pass.
	fill_list_kernel<<<di.sms * WINDOW_BLOCKS_PER_SM, 256, 0, s>>>(ws.frames.p, ws.state.p,
		ws.cands.p, &ws.ctl.p->n_holes);
	mark(rec, K_FILL);
}

static void launch_epilogue(Workspace &ws, const Layout &L, const DeviceInfo &di, cudaStream_t s,
	Recorder *rec = nullptr)
{
	if (!L.maxiter)
		return;
	const int nrows = (int)L.rows.size();
	restore_kernel<<<grid_for_rows(di, nrows, L.tune.row_blocks_per_sm), 256, 0, s>>>(ws.frames.p, ws.rows.p, nrows);
	mark(rec, K_RESTORE);
}

// Whole cleaning on stream s without graphs.
static void enqueue_plain(Workspace &ws, const Layout &L, const DeviceInfo &di, cudaStream_t s,
	Recorder *rec = nullptr)
{
	if (rec)
		rec->begin(s);
	launch_prologue(ws, L, di, s, rec);
	for (int it = 0; it < L.maxiter; ++it)
		launch_pass(ws, L, di, s, GraphLoop{}, it > 0, rec);
	launch_epilogue(ws, L, di, s, rec);
	check(cudaGetLastError());
}

// Status of one frame after a call: a kernel whose bounded wait ran out is a
// CUDA-level failure; a target without finite donors is the reference's
// "no finite replacement donors" (src/cleaner.cuh:95-96,137-138).
static void check_state(const FrameState &st)
{
	if (st.fault)
		throw std::runtime_error("a detection kernel gave up waiting for its copies");
	if (st.error || (st.holes && st.allowed && !st.finite))
		throw InvalidArgument("no finite replacement donors");
}

// Copy per-frame state back and turn it into a status (stream must be idle
// after this returns).
static void finish(Workspace &ws, size_t nf, cudaStream_t s, std::vector<int> *passes = nullptr)
{
	ws.hstate.ensure(nf);
	check(cudaMemcpyAsync(ws.hstate.p, ws.state.p, nf * sizeof(FrameState), cudaMemcpyDeviceToHost, s));
	check(cudaStreamSynchronize(s));
	check(cudaGetLastError());
	if (passes)
		passes->assign(nf, 0);
	for (size_t f = 0; f < nf; ++f) {
		const FrameState &st = ws.hstate.p[f];
		if (passes)
			(*passes)[f] = (int)st.passes;
		check_state(st);
	}
}

template <class F> static int guarded(F run, char *msg, size_t len)
{
	if (msg && len)
		msg[0] = 0;
	try {
		run();
		return CUSMIC_OK;
	} catch (const std::invalid_argument &e) {
		if (msg && len)
			std::snprintf(msg, len, "%s", e.what());
		return CUSMIC_INVALID;
	} catch (const std::bad_alloc &e) {
		if (msg && len)
			std::snprintf(msg, len, "%s", e.what());
		return CUSMIC_NO_MEMORY;
	} catch (const std::exception &e) {
		if (msg && len)
			std::snprintf(msg, len, "%s", e.what());
		return CUSMIC_CUDA_ERROR;
	} catch (...) {
		if (msg && len)
			std::snprintf(msg, len, "unknown error");
		return CUSMIC_CUDA_ERROR;
	}
}

static void run_device(const cusmic_image *ims, size_t nf, const cusmic_options &o,
	const cusmic_frame_scalars *sc, double *clean, uint8_t *mask, cudaStream_t s,
	std::vector<int> *passes = nullptr)
{
	check_device_alignment(ims, nf, clean);
	int dev;
	check(cudaGetDevice(&dev));
	DeviceInfo di = device_info(dev);
	Layout L = make_layout(ims, nf, o, sc, clean, mask, di);
	Lease ws(dev);
	upload(*ws, L, s);
	enqueue_plain(*ws, L, di, s);
	finish(*ws, nf, s, passes);
}

} // namespace cb

using namespace cb;

extern "C" const char *cusmic_version(void)
{
	return CUSMIC_B200_VERSION;
}

extern "C" int cusmic_cuda_version(void)
{
	return CUDART_VERSION;
}

extern "C" void cusmic_default_options(cusmic_options *options)
{
	if (options)
		*options = {3, 5, 3, NAN, 0, NAN, 4, CUSMIC_MIRROR};
}

extern "C" int remove_cosmics(const cusmic_image *im, const cusmic_options *o, double *clean,
	uint8_t *mask, char *msg, size_t len)
{
	return guarded([&] {
		check_arguments(im, 1, o, nullptr, clean, mask, true);
		const size_t n = im->width * im->height;

		int dev;
		check(cudaGetDevice(&dev));
		Lease ws(dev);
		const double *gmap = im->error ? nullptr : im->gain;
		const double *rnmap = im->error ? nullptr : im->readnoise;
		ws->hdata.ensure(n);
		ws->hclean.ensure(n);
		ws->hout.ensure(n);
		cudaStream_t s = nullptr;
		ws->stage_io.in(ws->hdata.p, im->data, n * sizeof(double), s);
		cusmic_image gpu = *im;
		gpu.data = ws->hdata.p;
		auto stage = [&](DevBuf<double> &b, const double *src) -> const double * {
			if (!src)
				return nullptr;
			b.ensure(n);
			ws->stage_io.in(b.p, src, n * sizeof(double), s);
			return b.p;
		};
		gpu.error = stage(ws->herror, im->error);
		gpu.gain = stage(ws->hgain, gmap);
		gpu.readnoise = stage(ws->hrn, rnmap);
		gpu.background = stage(ws->hbg, im->background);
		if (im->mask) {
			ws->hmask.ensure(n);
			ws->stage_io.in(ws->hmask.p, im->mask, n, s);
			gpu.mask = ws->hmask.p;
		}
		DeviceInfo di = device_info(dev);
		// The maps' contents are checked on the device (the reference checks
		// them on the host first, src/api.cu:161-168): the flags are read
		// before any output is copied back, so a failing call leaves the
		// outputs untouched and reports the first failing map, in the
		// reference's order.
		ws->hflags.ensure(1);
		check(cudaMemsetAsync(ws->hflags.p, 0, sizeof(unsigned), s));
		auto validate = [&](const double *p, int minimum, unsigned bit) {
			if (!p)
				return;
			const long long blocks = ((long long)n + 255) / 256 < di.sms * 4 ? ((long long)n + 255) / 256
											   : di.sms * 4;
			validate_kernel<<<(int)blocks, 256, 0, s>>>(p, (long long)n, minimum, ws->hflags.p, bit);
		};
		validate(gpu.error, 1, 1u);
		validate(gpu.gain, 1, 2u);
		validate(gpu.readnoise, 0, 4u);
		validate(gpu.background, -1, 8u);
		Layout L = make_layout(&gpu, 1, *o, nullptr, ws->hclean.p, ws->hout.p, di);
		upload(*ws, L, s);
		enqueue_plain(*ws, L, di, s);
		unsigned bad = 0;
		check(cudaMemcpyAsync(&bad, ws->hflags.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
		check(cudaStreamSynchronize(s));
		if (bad & 1u)
			throw InvalidArgument("error must be finite and positive");
		if (bad & 2u)
			throw InvalidArgument("gain must be finite and positive");
		if (bad & 4u)
			throw InvalidArgument("read noise must be finite and nonnegative");
		if (bad & 8u)
			throw InvalidArgument("background must be finite");
		finish(*ws, 1, s);
		ws->stage_io.out(clean, ws->hclean.p, n * sizeof(double), s);
		ws->stage_io.out(mask, ws->hout.p, n, s);
	}, msg, len);
}

extern "C" int remove_cosmics_batch_device(const cusmic_image *ims, size_t nf,
	const cusmic_options *o, double *clean, uint8_t *mask, void *stream, char *msg, size_t len)
{
	return guarded([&] {
		check_arguments(ims, nf, o, nullptr, clean, mask, true);
		run_device(ims, nf, *o, nullptr, clean, mask, (cudaStream_t)stream);
	}, msg, len);
}

extern "C" int remove_cosmics_device(const cusmic_image *im, const cusmic_options *o, double *clean,
	uint8_t *mask, void *stream, char *msg, size_t len)
{
	return remove_cosmics_batch_device(im, 1, o, clean, mask, stream, msg, len);
}

extern "C" int cusmic_ragged_batch_device(const cusmic_image *ims, size_t nf,
	const cusmic_options *o, const cusmic_frame_scalars *sc, double *clean, uint8_t *mask,
	void *stream, char *msg, size_t len)
{
	return guarded([&] {
		check_arguments(ims, nf, o, sc, clean, mask, false);
		run_device(ims, nf, *o, sc, clean, mask, (cudaStream_t)stream);
	}, msg, len);
}

// ---------------------------------------------------------------------------
// Host-buffer batch.  The reference's host entry point cleans one frame and
// moves its maps and pixels with blocking copies (src/api.cu:116-153); a
// batch of frames called that way pays every map again per frame and never
// overlaps a frame's inbound copy with the previous frame's outbound copy.
// Here frames are cleaned in chunks of whole frames on three streams: chunk
// k + 1's pixels go up while chunk k is cleaned and chunk k - 1's results
// come down (PCIe moves both directions at once), and a map that several
// frames share is uploaded and checked once per call.

namespace cb {

constexpr size_t HB_CHUNK_BYTES = size_t(64) << 20; // input bytes a chunk aims for
constexpr size_t HB_ALIGN = 16;                     // pixels: chunk offsets stay 16-byte aligned

static size_t hb_round(size_t n)
{
	return (n + HB_ALIGN - 1) / HB_ALIGN * HB_ALIGN;
}

// The map-check flags of validate_kernel, in the reference's order of checks
// (src/api.cu:161-168).
static void throw_map_flags(unsigned bad)
{
	if (bad & 1u)
		throw InvalidArgument("error must be finite and positive");
	if (bad & 2u)
		throw InvalidArgument("gain must be finite and positive");
	if (bad & 4u)
		throw InvalidArgument("read noise must be finite and nonnegative");
	if (bad & 8u)
		throw InvalidArgument("background must be finite");
}

// Streams and events of one call; on every exit (an exception included) it
// waits for the copies in flight, so none touches the caller's buffers after
// the call returns.
struct HostPipe {
	cudaStream_t h2d = nullptr, comp = nullptr, d2h = nullptr;
	std::vector<cudaEvent_t> in; // per chunk: its inputs are on the device
	cudaEvent_t done[2] = {}, out[2] = {}, shared = nullptr;
	explicit HostPipe(size_t chunks) : in(chunks, nullptr)
	{
		check(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
		check(cudaStreamCreateWithFlags(&comp, cudaStreamNonBlocking));
		check(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
		for (cudaEvent_t &e : in)
			check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
		for (int i = 0; i < 2; ++i) {
			check(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
			check(cudaEventCreateWithFlags(&out[i], cudaEventDisableTiming));
		}
		check(cudaEventCreateWithFlags(&shared, cudaEventDisableTiming));
	}
	~HostPipe()
	{
		for (cudaStream_t s : {h2d, comp, d2h})
			if (s) {
				cudaStreamSynchronize(s);
				cudaStreamDestroy(s);
			}
		for (cudaEvent_t e : in)
			if (e)
				cudaEventDestroy(e);
		for (int i = 0; i < 2; ++i)
			for (cudaEvent_t e : {done[i], out[i]})
				if (e)
					cudaEventDestroy(e);
		if (shared)
			cudaEventDestroy(shared);
	}
};

// Host copies of a call running on the copy threads; waited for on every
// exit, so none writes into the caller's buffers after the call returns.
struct HostCopies {
	std::vector<std::unique_ptr<CopyPool::Join>> join;
	explicit HostCopies(size_t n) : join(n) {}
	~HostCopies()
	{
		for (auto &j : join)
			if (j)
				CopyPool::wait(*j);
	}
};

static void run_host_batch(const cusmic_image *ims, size_t nf, const cusmic_options &o,
	const cusmic_frame_scalars *sc, double *clean, uint8_t *mask)
{
	int dev;
	check(cudaGetDevice(&dev));
	const DeviceInfo di = device_info(dev);
	// A host map used by more than one frame is shared: uploaded once.
	std::map<const void *, int> uses;
	auto model_map = [](const cusmic_image &im, const double *p) { return im.error ? nullptr : p; };
	for (size_t f = 0; f < nf; ++f) {
		const cusmic_image &im = ims[f];
		for (const void *p : {(const void *)im.error, (const void *)model_map(im, im.gain),
			     (const void *)model_map(im, im.readnoise), (const void *)im.background,
			     (const void *)im.mask})
			if (p)
				++uses[p];
	}
	auto is_shared = [&](const void *p) { return p && uses[p] > 1; };
	// Each shared map: its pixels (the largest frame that reads it), its
	// check (validate_kernel's minimum and flag; mask: none) and its offset in
	// the shared buffer of its type.
	struct SharedMap {
		size_t n = 0, off = 0;
		int minimum = 0;
		unsigned bit = 0; // 0: a mask
	};
	std::map<const void *, SharedMap> shared;
	for (size_t f = 0; f < nf; ++f) {
		const cusmic_image &im = ims[f];
		const size_t n = im.width * im.height;
		const struct {
			const void *p;
			int minimum;
			unsigned bit;
		} maps[] = {{im.error, 1, 1u}, {model_map(im, im.gain), 1, 2u},
			{model_map(im, im.readnoise), 0, 4u}, {im.background, -1, 8u}, {im.mask, 0, 0u}};
		for (const auto &m : maps)
			if (is_shared(m.p)) {
				SharedMap &e = shared[m.p];
				e.n = std::max(e.n, n);
				e.minimum = m.minimum;
				e.bit = m.bit;
			}
	}
	size_t shared_px = 0, shared_mask_px = 0;
	for (auto &e : shared) {
		size_t &end = e.second.bit ? shared_px : shared_mask_px;
		e.second.off = end;
		end += hb_round(e.second.n);
	}
	// Chunks of consecutive frames: input bytes up to HB_CHUNK_BYTES, at
	// least one frame.
	std::vector<size_t> first{0};
	size_t bytes = 0, chunk_px = 0, max_px = 0;
	for (size_t f = 0; f < nf; ++f) {
		const cusmic_image &im = ims[f];
		const size_t n = im.width * im.height;
		size_t fb = 8 * n;
		for (const double *p : {im.error, model_map(im, im.gain), model_map(im, im.readnoise),
			     im.background})
			fb += p && !is_shared(p) ? 8 * n : 0;
		fb += im.mask && !is_shared(im.mask) ? n : 0;
		if (f > first.back() && bytes + fb > HB_CHUNK_BYTES) {
			first.push_back(f);
			bytes = chunk_px = 0;
		}
		bytes += fb;
		chunk_px += hb_round(n);
		max_px = std::max(max_px, chunk_px);
	}
	first.push_back(nf);
	const size_t nchunks = first.size() - 1;
	// A chunk whose frames have no background returns sparsely: without a
	// background every output pixel outside the mask equals its input bit
	// for bit (prepare copies it, restore writes holes back), so host threads
	// copy the inputs to the outputs and only the flagged pixels' values and
	// positions cross PCIe (16 bytes per flagged pixel instead of 9 per
	// pixel).
	std::vector<char> sparse(nchunks, 1);
	bool any_sparse = false;
	for (size_t k = 0; k < nchunks; ++k) {
		for (size_t f = first[k]; f < first[k + 1]; ++f)
			if (ims[f].background || !std::isnan(scalars_for(o, sc, f).bg))
				sparse[k] = 0;
		any_sparse |= sparse[k] != 0;
	}
	std::vector<size_t> out_off(nf + 1, 0); // first output pixel of each frame
	for (size_t f = 0; f < nf; ++f)
		out_off[f + 1] = out_off[f] + ims[f].width * ims[f].height;

	bool any[5] = {}; // per-frame (not shared) maps present: error, gain, rn, bg, mask
	for (size_t f = 0; f < nf; ++f) {
		const cusmic_image &im = ims[f];
		any[0] |= im.error && !is_shared(im.error);
		any[1] |= model_map(im, im.gain) && !is_shared(im.gain);
		any[2] |= model_map(im, im.readnoise) && !is_shared(im.readnoise);
		any[3] |= im.background && !is_shared(im.background);
		any[4] |= im.mask && !is_shared(im.mask);
	}
	// Inputs go through a device ring of `slots` chunk slots.  When the whole
	// call's inputs fit a quarter of the free device memory (at most
	// 16 GiB) the ring holds every chunk, and every inbound copy is queued at
	// the start; otherwise a slot is refilled as soon as its chunk is cleaned.
	const size_t px_bytes = 8 + 8 * (any[0] + any[1] + any[2] + any[3]) + any[4];
	size_t free_b = 0, total_b = 0;
	check(cudaMemGetInfo(&free_b, &total_b));
	const size_t budget = std::min(free_b / 4, size_t(16) << 30);
	const size_t slots = std::max<size_t>(2, std::min(nchunks, budget / std::max<size_t>(1, max_px * px_bytes)));
	Lease wl[2] = {Lease(dev), Lease(dev)};
	Workspace *ws[2] = {&*wl[0], &*wl[1]};
	Workspace &ring = *ws[0]; // the input ring and the shared maps
	ring.hdata.ensure(slots * max_px);
	if (any[0])
		ring.herror.ensure(slots * max_px);
	if (any[1])
		ring.hgain.ensure(slots * max_px);
	if (any[2])
		ring.hrn.ensure(slots * max_px);
	if (any[3])
		ring.hbg.ensure(slots * max_px);
	if (any[4])
		ring.hmask.ensure(slots * max_px);
	for (Workspace *w : ws) {
		w->hclean.ensure(max_px);
		w->hout.ensure(max_px);
		w->hflags.ensure(2); // one 8-byte word: the flags and padding
		w->hflags_host.ensure(2);
		w->hcount.ensure(1);
		if (any_sparse && o.maxiter)
			w->hsp_val.ensure(max_px);
	}
	if (shared_px)
		ring.hshared.ensure(shared_px);
	if (shared_mask_px)
		ring.hshared_mask.ensure(shared_mask_px);
	HostPipe pipe(nchunks);
	HostCopies host(nchunks);
	auto up = [&](void *dst, const void *src, size_t n) {
		if (HostStage::pinned(src))
			check(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, pipe.h2d));
		else
			ring.stage_io.in(dst, src, n, pipe.h2d);
	};
	auto validate = [&](const double *p, long long n, int minimum, unsigned *flags, unsigned bit) {
		const long long blocks = (n + 255) / 256 < di.sms * 4 ? (n + 255) / 256 : di.sms * 4;
		validate_kernel<<<(int)blocks, 256, 0, pipe.comp>>>(p, n, minimum, flags, bit);
	};
	// Shared maps first (on the inbound stream, ahead of every chunk).
	for (const auto &e : shared) {
		if (e.second.bit)
			up(ring.hshared.p + e.second.off, e.first, e.second.n * sizeof(double));
		else
			up(ring.hshared_mask.p + e.second.off, e.first, e.second.n);
	}
	check(cudaEventRecord(pipe.shared, pipe.h2d));
	// The host side of the sparse chunks (outputs = inputs, masks zero) runs
	// on the copy threads from the start, in chunk order.
	for (size_t k = 0; k < nchunks; ++k)
		if (sparse[k]) {
			host.join[k].reset(new CopyPool::Join);
			for (size_t f = first[k]; f < first[k + 1]; ++f) {
				const size_t np = ims[f].width * ims[f].height;
				if (clean + out_off[f] != ims[f].data)
					CopyPool::get().submit(*host.join[k], clean + out_off[f], ims[f].data,
						np * sizeof(double));
				CopyPool::get().submit(*host.join[k], mask + out_off[f], nullptr, np);
			}
		}

	std::vector<cusmic_image> dims(nf);
	auto issue_inputs = [&](size_t k) {
		size_t off = (k % slots) * max_px;
		for (size_t f = first[k]; f < first[k + 1]; ++f) {
			const cusmic_image &im = ims[f];
			const size_t n = im.width * im.height;
			cusmic_image &d = dims[f];
			d = im;
			d.data = ring.hdata.p + off;
			up(ring.hdata.p + off, im.data, n * sizeof(double));
			auto place = [&](const double *p, DevBuf<double> &b) -> const double * {
				if (!p)
					return nullptr;
				if (is_shared(p))
					return ring.hshared.p + shared[p].off;
				up(b.p + off, p, n * sizeof(double));
				return b.p + off;
			};
			d.error = place(im.error, ring.herror);
			d.gain = place(model_map(im, im.gain), ring.hgain);
			d.readnoise = place(model_map(im, im.readnoise), ring.hrn);
			d.background = place(im.background, ring.hbg);
			if (im.mask) {
				if (is_shared(im.mask)) {
					d.mask = ring.hshared_mask.p + shared[im.mask].off;
				} else {
					up(ring.hmask.p + off, im.mask, n);
					d.mask = ring.hmask.p + off;
				}
			}
			off += hb_round(n);
		}
		check(cudaEventRecord(pipe.in[k], pipe.h2d));
	};
	auto finish_chunk = [&](size_t k) {
		Workspace &w = *ws[k & 1];
		check(cudaEventSynchronize(pipe.done[k & 1]));
		throw_map_flags(*w.hflags_host.p);
		for (size_t f = first[k]; f < first[k + 1]; ++f)
			check_state(w.hstate.p[f - first[k]]);
		check(cudaStreamWaitEvent(pipe.d2h, pipe.done[k & 1], 0));
		if (sparse[k]) {
			const size_t n = o.maxiter ? (size_t)*w.hcount.p : 0;
			if (n) {
				w.hsp_idx_host.ensure(n);
				w.hsp_val_host.ensure(n);
				check(cudaMemcpyAsync(w.hsp_idx_host.p, w.targets.p, n * sizeof(uint2),
					cudaMemcpyDeviceToHost, pipe.d2h));
				check(cudaMemcpyAsync(w.hsp_val_host.p, w.hsp_val.p, n * sizeof(double),
					cudaMemcpyDeviceToHost, pipe.d2h));
			}
			check(cudaEventRecord(pipe.out[k & 1], pipe.d2h));
			CopyPool::wait(*host.join[k]); // outputs = inputs, masks zero
			check(cudaEventSynchronize(pipe.out[k & 1]));
			for (size_t i = 0; i < n; ++i) {
				const uint2 t = w.hsp_idx_host.p[i];
				const size_t at = out_off[first[k] + t.x] + t.y;
				clean[at] = w.hsp_val_host.p[i];
				mask[at] = 1;
			}
			return;
		}
		size_t off = 0;
		for (size_t f = first[k]; f < first[k + 1]; ++f) {
			const size_t n = ims[f].width * ims[f].height;
			for (int part = 0; part < 2; ++part) {
				void *dst = part ? (void *)(mask + out_off[f]) : (void *)(clean + out_off[f]);
				const void *src = part ? (const void *)(w.hout.p + off) : (const void *)(w.hclean.p + off);
				const size_t len = part ? n : n * sizeof(double);
				if (HostStage::pinned(dst))
					check(cudaMemcpyAsync(dst, src, len, cudaMemcpyDeviceToHost, pipe.d2h));
				else
					w.stage_io.out(dst, src, len, pipe.d2h);
			}
			off += n;
		}
		check(cudaEventRecord(pipe.out[k & 1], pipe.d2h));
	};
	for (size_t k = 0; k < std::min(slots, nchunks); ++k)
		issue_inputs(k);
	for (size_t k = 0; k < nchunks; ++k) {
		Workspace &w = *ws[k & 1];
		const size_t f0 = first[k], f1 = first[k + 1], nc = f1 - f0;
		// Clean the chunk once its inputs are up and its slot's outputs of
		// chunk k - 2 are down.
		check(cudaStreamWaitEvent(pipe.comp, pipe.in[k], 0));
		if (k >= 2)
			check(cudaStreamWaitEvent(pipe.comp, pipe.out[k & 1], 0));
		check(cudaMemsetAsync(w.hflags.p, 0, 2 * sizeof(unsigned), pipe.comp));
		if (k == 0) { // the shared maps are checked with the first chunk
			check(cudaStreamWaitEvent(pipe.comp, pipe.shared, 0));
			for (const auto &e : shared)
				if (e.second.bit)
					validate(ring.hshared.p + e.second.off, (long long)e.second.n,
						e.second.minimum, w.hflags.p, e.second.bit);
		}
		for (size_t f = f0; f < f1; ++f) {
			const cusmic_image &im = ims[f], &d = dims[f];
			const long long n = (long long)(im.width * im.height);
			if (im.error && !is_shared(im.error))
				validate(d.error, n, 1, w.hflags.p, 1u);
			if (d.gain && !is_shared(im.gain))
				validate(d.gain, n, 1, w.hflags.p, 2u);
			if (d.readnoise && !is_shared(im.readnoise))
				validate(d.readnoise, n, 0, w.hflags.p, 4u);
			if (im.background && !is_shared(im.background))
				validate(d.background, n, -1, w.hflags.p, 8u);
		}
		Layout L = make_layout(dims.data() + f0, nc, o, sc ? sc + f0 : nullptr, w.hclean.p,
			w.hout.p, di);
		upload(w, L, pipe.comp, true);
		enqueue_plain(w, L, di, pipe.comp);
		if (sparse[k] && o.maxiter)
			gather_targets_kernel<<<di.sms * 4, 256, 0, pipe.comp>>>(w.frames.p, w.targets.p,
				&w.ctl.p->n_targets, w.hsp_val.p);
		// The chunk's status into page-locked memory, written by a kernel
		// (a copy would queue behind the outbound copies of earlier chunks).
		w.hstate.ensure(nc);
		static_assert(sizeof(FrameState) % 8 == 0, "8-byte words");
		WordCopies st{};
		st.part[0] = WordCopy{reinterpret_cast<const unsigned long long *>(w.state.p),
			static_cast<unsigned long long *>(const_cast<void *>(host_device_ptr(w.hstate.p))),
			(long long)(nc * sizeof(FrameState) / 8)};
		st.part[1] = WordCopy{&w.ctl.p->n_targets,
			static_cast<unsigned long long *>(const_cast<void *>(host_device_ptr(w.hcount.p))), 1};
		st.part[2] = WordCopy{reinterpret_cast<const unsigned long long *>(w.hflags.p),
			static_cast<unsigned long long *>(const_cast<void *>(host_device_ptr(w.hflags_host.p))), 1};
		st.n = 3;
		word_copy_kernel<<<1, 256, 0, pipe.comp>>>(st);
		check(cudaEventRecord(pipe.done[k & 1], pipe.comp));
		if (k >= 1) {
			finish_chunk(k - 1);
			// Chunk k - 1 is cleaned: its input slot takes chunk k - 1 + slots.
			if (k - 1 + slots < nchunks)
				issue_inputs(k - 1 + slots);
		}
	}
	finish_chunk(nchunks - 1);
	check(cudaStreamSynchronize(pipe.d2h));
	check(cudaGetLastError());
}

} // namespace cb

extern "C" int cusmic_batch_host(const cusmic_image *ims, size_t nf, const cusmic_options *o,
	const cusmic_frame_scalars *sc, double *clean, uint8_t *mask, char *msg, size_t len)
{
	return guarded([&] {
		check_arguments(ims, nf, o, sc, clean, mask, false);
		run_host_batch(ims, nf, *o, sc, clean, mask);
	}, msg, len);
}

// ---------------------------------------------------------------------------
// Plans: a fixed batch with its own workspace, descriptors uploaded once, and
// optionally the whole cleaning captured as one CUDA graph.  The maxiter loop
// becomes a conditional WHILE node whose condition control_kernel sets from
// the device (any frame still active and passes left), so the early exit costs
// no host round trip.

struct cusmic_plan {
	int device = -1;
	int flags = 0;
	Layout L;
	DeviceInfo di;
	Workspace ws;
	cusmic_options options{};
	std::vector<cusmic_image> ims;
	std::vector<cusmic_frame_scalars> scalars;
	cudaStream_t private_stream = nullptr;
	cudaStream_t last = nullptr;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	bool executed = false;

	~cusmic_plan()
	{
		if (exec)
			cudaGraphExecDestroy(exec);
		if (graph)
			cudaGraphDestroy(graph);
		if (private_stream)
			cudaStreamDestroy(private_stream);
	}
};

namespace cb {

static void capture_graph(cusmic_plan &p)
{
	cudaStream_t cs = p.private_stream;
	check(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
	try {
		launch_prologue(p.ws, p.L, p.di, cs);
		if (p.L.maxiter) {
			cudaStreamCaptureStatus st;
			cudaGraph_t g;
			const cudaGraphNode_t *deps = nullptr;
			size_t nd = 0;
			check(cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd));
			// The full first pass sets the loop condition (its control
			// kernel runs upstream of the while node); the body repeats the
			// incremental pass.
			cudaGraphConditionalHandle handle;
			check(cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
			launch_pass(p.ws, p.L, p.di, cs, GraphLoop{handle, true}, false);
			check(cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd));
			cudaGraphNodeParams cp = {};
			cp.type = cudaGraphNodeTypeConditional;
			cp.conditional.handle = handle;
			cp.conditional.type = cudaGraphCondTypeWhile;
			cp.conditional.size = 1;
			cudaGraphNode_t node;
			check(cudaGraphAddNode(&node, g, deps, nd, &cp));
			cudaGraph_t body = cp.conditional.phGraph_out[0];
			check(cudaStreamUpdateCaptureDependencies(cs, &node, 1,
				cudaStreamSetCaptureDependencies));
			cudaStream_t bs;
			check(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
			cudaError_t err = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0,
				cudaStreamCaptureModeThreadLocal);
			if (err == cudaSuccess) {
				launch_pass(p.ws, p.L, p.di, bs, GraphLoop{handle, true}, true);
				err = cudaStreamEndCapture(bs, nullptr);
			}
			cudaStreamDestroy(bs);
			check(err);
		}
		launch_epilogue(p.ws, p.L, p.di, cs);
	} catch (...) {
		cudaGraph_t g = nullptr;
		cudaStreamEndCapture(cs, &g);
		if (g)
			cudaGraphDestroy(g);
		throw;
	}
	check(cudaStreamEndCapture(cs, &p.graph));
	check(cudaGraphInstantiate(&p.exec, p.graph, 0));
}

static void plan_upload(cusmic_plan &p)
{
	upload(p.ws, p.L, p.private_stream);
	check(cudaStreamSynchronize(p.private_stream));
}

} // namespace cb

extern "C" int cusmic_plan_create(cusmic_plan **out, const cusmic_image *ims, size_t nf,
	const cusmic_options *o, const cusmic_frame_scalars *sc, double *clean, uint8_t *mask,
	int flags, char *msg, size_t len)
{
	return guarded([&] {
		if (!out)
			throw InvalidArgument("invalid plan pointer");
		*out = nullptr;
		check_arguments(ims, nf, o, sc, clean, mask, false);
		check_device_alignment(ims, nf, clean);
		std::unique_ptr<cusmic_plan> p(new cusmic_plan);
		check(cudaGetDevice(&p->device));
		p->flags = flags;
		p->di = device_info(p->device);
		p->options = *o;
		p->ims.assign(ims, ims + nf);
		if (sc)
			p->scalars.assign(sc, sc + nf);
		p->L = make_layout(ims, nf, *o, sc, clean, mask, p->di);
		check(cudaStreamCreateWithFlags(&p->private_stream, cudaStreamNonBlocking));
		plan_upload(*p);
		if (flags & CUSMIC_PLAN_GRAPH)
			capture_graph(*p);
		*out = p.release();
	}, msg, len);
}

extern "C" int cusmic_plan_bind(cusmic_plan *p, const cusmic_image *ims, double *clean,
	uint8_t *mask, char *msg, size_t len)
{
	return guarded([&] {
		if (!p || !ims || !clean || !mask)
			throw InvalidArgument("invalid plan or buffers");
		const size_t nf = p->ims.size();
		for (size_t f = 0; f < nf; ++f) {
			const cusmic_image &a = ims[f], &b = p->ims[f];
			if (!a.data || a.width != b.width || a.height != b.height ||
				!a.error != !b.error || !a.gain != !b.gain || !a.readnoise != !b.readnoise ||
				!a.background != !b.background || !a.mask != !b.mask)
				throw InvalidArgument("frames must keep the plan's shapes and maps");
		}
		if (p->last)
			check(cudaStreamSynchronize(p->last));
		Layout L = make_layout(ims, nf, p->options, p->scalars.empty() ? nullptr : p->scalars.data(),
			clean, mask, p->di);
		// The plan's threshold blocks are fixed: frames must keep their
		// sharing of error maps.
		check_device_alignment(ims, nf, clean);
		if (L.thr_base != p->L.thr_base)
			throw InvalidArgument("rebound frames must keep the plan's sharing of error maps");
		for (size_t f = 0; f < nf; ++f) {
			L.frames[f].bits = p->L.frames[f].bits;
			L.frames[f].floors = p->L.frames[f].floors;
			L.frames[f].rowcand = p->L.frames[f].rowcand;
			L.frames[f].rowchg = p->L.frames[f].rowchg;
			L.frames[f].sig_raw = p->L.frames[f].sig_raw;
			L.frames[f].noise = p->L.frames[f].noise;
			L.frames[f].out = L.frames[f].clean; // the new output buffer
			if (p->L.frames[f].out != p->L.frames[f].clean) // working pixels in the workspace
				L.frames[f].clean = p->L.frames[f].clean;
		}
		p->ims.assign(ims, ims + nf);
		p->L.frames = L.frames;
		// New buffers can change which prepare kernels suit the batch: the
		// graph is captured again with the new choice.
		const bool recapture = L.prep_bulk != p->L.prep_bulk || L.fused != p->L.fused;
		p->L.prep_bulk = L.prep_bulk;
		p->L.fused = L.fused;
		const size_t bytes = nf * sizeof(FrameDesc);
		std::memcpy(p->ws.stage.p, p->L.frames.data(), bytes);
		check(cudaMemcpyAsync(p->ws.frames.p, p->ws.stage.p, bytes, cudaMemcpyHostToDevice,
			p->private_stream));
		check(cudaStreamSynchronize(p->private_stream));
		if (recapture && p->exec) {
			cudaGraphExecDestroy(p->exec);
			cudaGraphDestroy(p->graph);
			p->exec = nullptr;
			p->graph = nullptr;
			capture_graph(*p);
		}
	}, msg, len);
}

extern "C" int cusmic_plan_execute(cusmic_plan *p, void *stream, char *msg, size_t len)
{
	return guarded([&] {
		if (!p)
			throw InvalidArgument("invalid plan");
		cudaStream_t s = (cudaStream_t)stream;
		if (p->exec)
			check(cudaGraphLaunch(p->exec, s));
		else
			enqueue_plain(p->ws, p->L, p->di, s);
		const size_t nf = p->L.frames.size();
		p->ws.hstate.ensure(nf);
		check(cudaMemcpyAsync(p->ws.hstate.p, p->ws.state.p, nf * sizeof(FrameState),
			cudaMemcpyDeviceToHost, s));
		p->last = s;
		p->executed = true;
	}, msg, len);
}

extern "C" int cusmic_plan_wait(cusmic_plan *p, char *msg, size_t len)
{
	return guarded([&] {
		if (!p || !p->executed)
			throw InvalidArgument("plan has not been executed");
		check(cudaStreamSynchronize(p->last));
		check(cudaGetLastError());
		for (size_t f = 0; f < p->L.frames.size(); ++f) {
			check_state(p->ws.hstate.p[f]);
		}
	}, msg, len);
}

extern "C" int cusmic_plan_passes(cusmic_plan *p, int *passes)
{
	if (!p || !passes || !p->executed)
		return CUSMIC_INVALID;
	if (cudaStreamSynchronize(p->last) != cudaSuccess)
		return CUSMIC_CUDA_ERROR;
	for (size_t f = 0; f < p->L.frames.size(); ++f)
		passes[f] = (int)p->ws.hstate.p[f].passes;
	return CUSMIC_OK;
}

extern "C" void cusmic_plan_destroy(cusmic_plan *p)
{
	if (!p)
		return;
	if (p->last)
		cudaStreamSynchronize(p->last);
	delete p;
}

extern "C" int cusmic_plan_profile(cusmic_plan *p, void *stream, double *ms, int *launches,
	int kinds, char *msg, size_t len)
{
	return guarded([&] {
		if (!p || !ms || !launches || kinds < K_KINDS)
			throw InvalidArgument("invalid plan or profile buffers");
		cudaStream_t s = (cudaStream_t)stream;
		Recorder rec;
		enqueue_plain(p->ws, p->L, p->di, s, &rec);
		const size_t nf = p->L.frames.size();
		p->ws.hstate.ensure(nf);
		check(cudaMemcpyAsync(p->ws.hstate.p, p->ws.state.p, nf * sizeof(FrameState),
			cudaMemcpyDeviceToHost, s));
		p->last = s;
		p->executed = true;
		check(cudaStreamSynchronize(s));
		for (int k = 0; k < kinds; ++k) {
			ms[k] = 0;
			launches[k] = 0;
		}
		for (size_t i = 1; i < rec.events.size(); ++i) {
			float t = 0;
			check(cudaEventElapsedTime(&t, rec.events[i - 1], rec.events[i]));
			ms[rec.kinds[i]] += t;
			launches[rec.kinds[i]] += 1;
		}
	}, msg, len);
}

extern "C" int cusmic_plan_backward(cusmic_plan *p, const double *grad_clean, double *grad_data,
	double *grad_background, void *stream, char *msg, size_t len)
{
	return guarded([&] {
		if (!p || !grad_clean || !grad_data)
			throw InvalidArgument("invalid plan or gradient buffers");
		if (!p->executed)
			throw InvalidArgument("plan has not been executed");
		check(cudaStreamSynchronize(p->last));
		const size_t nf = p->L.frames.size();
		for (size_t f = 0; f < nf; ++f) {
			check_state(p->ws.hstate.p[f]);
		}
		bool map_mode = false;
		for (const FrameDesc &d : p->L.frames)
			map_mode |= d.bg_map != nullptr;
		cudaStream_t s = (cudaStream_t)stream;
		const Layout &L = p->L;
		const int nrows = (int)L.rows.size();
		if (grad_background && !map_mode)
			check(cudaMemsetAsync(grad_background, 0, nf * sizeof(double), s));
		if (!L.maxiter) {
			// Zero iterations: out = (x + bg) - bg everywhere, an identity.
			check(cudaMemcpyAsync(grad_data, grad_clean, L.total_px * sizeof(double),
				cudaMemcpyDeviceToDevice, s));
			if (grad_background && map_mode)
				check(cudaMemsetAsync(grad_background, 0, L.total_px * sizeof(double), s));
		} else {
			bwd_dense_kernel<<<grid_for_rows(p->di, nrows), 256, 0, s>>>(p->ws.frames.p,
				p->ws.rows.p, nrows, grad_clean, grad_data, map_mode ? grad_background : nullptr,
				p->ws.offsets.p);
			bwd_scatter_kernel<<<p->di.sms * 8, 256, 0, s>>>(p->ws.frames.p, p->ws.targets.p,
				&p->ws.ctl.p->n_targets, p->ws.offsets.p, grad_clean, grad_data,
				map_mode ? grad_background : nullptr, map_mode ? nullptr : grad_background);
		}
		check(cudaGetLastError());
		check(cudaStreamSynchronize(s));
	}, msg, len);
}

// ---------------------------------------------------------------------------
// Allocation-free single-frame entry point.
//
// Some callers cannot allocate device memory at the moment they clean a frame:
// a real-time acquisition loop that allows allocation only at start-up
// (cudaMalloc can block for milliseconds and cudaFree synchronises the whole
// device), or a process whose own caching allocator has already reserved the
// GPU's memory, so a cudaMalloc here would fail.  For them this entry point
// keeps all of its scratch (descriptor, per-frame state, loop control, work
// lists, bit planes and target/candidate/seed lists) in the static device
// array below.  Every GPU that loads this library holds the array until the
// process exits.  Calls share it and it keeps the last call's contents, so
// every call clears what must start at zero; two calls whose work overlaps on
// the GPU race, so callers serialise them (one stream, or their own ordering).

namespace cb {

constexpr size_t NOALLOC_MAX_PIXELS = 512 * 512;
constexpr int NOALLOC_MAX_ROWS = 16384;
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(12) << 20; // 12 MiB

static __device__ __align__(256) unsigned char noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Offsets of the scratch segments for a w x h frame (256-byte aligned).
struct NoallocLayout {
	size_t desc, state, ctl, offsets, rows, items, bits, targets, cands, seeds, end;
	int nitems;
	long long plane;
};

static NoallocLayout noalloc_layout(int w, int h, bool error_map)
{
	auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
	NoallocLayout L{};
	const size_t n = (size_t)w * h;
	const int words = (w + 31) / 32;
	const int rows_per_item = error_map ? STREAM_ROWS : MTILE;
	L.nitems = ((w + 31) / 32) * ((h + rows_per_item - 1) / rows_per_item);
	L.plane = (long long)h * words;
	size_t o = 0;
	L.desc = o;
	o = up(o + sizeof(FrameDesc));
	L.state = o;
	o = up(o + sizeof(FrameState));
	L.ctl = o;
	o = up(o + sizeof(Control));
	L.offsets = o;
	o = up(o + sizeof(long long));
	L.rows = o;
	o = up(o + (size_t)h * sizeof(int2));
	L.items = o;
	o = up(o + (size_t)L.nitems * sizeof(int4));
	L.bits = o;
	o = up(o + (size_t)N_PLANES * L.plane * sizeof(uint32_t));
	L.targets = o;
	o = up(o + n * sizeof(uint2));
	L.cands = o;
	o = up(o + n * sizeof(uint2));
	L.seeds = o;
	o = up(o + n * sizeof(Seed));
	L.end = o;
	return L;
}

// Writes the frame descriptor, its row list and its strip (or tile) list
// into the scratch, so the call needs no host-side staging buffer.
__global__ void noalloc_setup_kernel(FrameDesc fd, FrameDesc *desc, long long *offsets, int2 *rows,
	int4 *items, int nitems, int rows_per_item)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i == 0) {
		*desc = fd;
		*offsets = 0;
	}
	if (i < fd.h)
		rows[i] = make_int2(0, i);
	if (i < nitems) {
		const int tx = (fd.w + 31) / 32;
		items[i] = make_int4(0, (i % tx) * 32, (i / tx) * rows_per_item, 0);
	}
}

struct NoallocDevice {
	unsigned char *scratch = nullptr;
	int sms = 0;
};

// Once per device, with that device current: the device address of the
// static array (its host-side name is only a stand-in) and the SM count.
static NoallocDevice noalloc_device(int dev)
{
	static std::mutex mu;
	static NoallocDevice cache[64];
	if (dev < 0 || dev >= 64)
		throw std::runtime_error("device ordinal out of range");
	std::lock_guard<std::mutex> lock(mu);
	NoallocDevice &d = cache[dev];
	if (!d.scratch) {
		void *ptr = nullptr;
		check(cudaGetSymbolAddress(&ptr, noalloc_scratch));
		check(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
		d.scratch = static_cast<unsigned char *>(ptr);
	}
	return d;
}

} // namespace cb

extern "C" int cusmic_set_tuning(const cusmic_tuning *table, size_t n, char *msg, size_t len)
{
	return guarded([&] {
		if (n && !table)
			throw InvalidArgument("invalid tuning table");
		for (size_t i = 0; i < n; ++i) {
			const cusmic_tuning &t = table[i];
			if (!(t.dense_rows == 0 || t.dense_rows == 4 || t.dense_rows == 8 || t.dense_rows == 16 ||
				    t.dense_rows == 32) ||
				t.dense_blocks_per_sm < 1 || t.dense_blocks_per_sm > BK_BLOCKS_PER_SM ||
				t.sparse_blocks_per_sm < 1 || t.sparse_blocks_per_sm > 8 ||
				t.row_blocks_per_sm < 1 || t.row_blocks_per_sm > 8)
				throw InvalidArgument("invalid tuning entry");
		}
		std::lock_guard<std::mutex> lock(tuning_mu);
		tuning_table.assign(table, table + n);
	}, msg, len);
}

extern "C" int cusmic_inject_fault(int what, long long value)
{
	switch (what) {
	case CUSMIC_FAULT_PREPARE_WAIT:
	case CUSMIC_FAULT_DETECT_WAIT:
		inject_wait[what - CUSMIC_FAULT_PREPARE_WAIT].store(value > 0 ? value : 0);
		return CUSMIC_OK;
	case CUSMIC_FAULT_NO_MEMORY:
		inject_alloc_failures.store(value > 0 ? value : 0);
		return CUSMIC_OK;
	default:
		return CUSMIC_INVALID;
	}
}

extern "C" int cusmic_get_tuning(size_t total_pixels, cusmic_tuning *out)
{
	if (!out)
		return CUSMIC_INVALID;
	*out = tuning_for(total_pixels);
	return CUSMIC_OK;
}

extern "C" int remove_cosmics_device_noalloc(const cusmic_image *im, const cusmic_options *o,
	double *clean, uint8_t *mask, void *stream, char *msg, size_t len)
{
	return guarded([&] {
		check_arguments(im, 1, o, nullptr, clean, mask, true);
		check_device_alignment(im, 1, clean);
		if (im->width * im->height > NOALLOC_MAX_PIXELS || im->height > (size_t)NOALLOC_MAX_ROWS)
			throw InvalidArgument("frame exceeds the static scratch: at most 262144 pixels "
				"and 16384 rows");
		int dev;
		check(cudaGetDevice(&dev));
		const NoallocDevice nd = noalloc_device(dev);
		cudaStream_t s = (cudaStream_t)stream;
		const int w = (int)im->width, h = (int)im->height;
		const bool error_map = im->error != nullptr;
		const NoallocLayout L = noalloc_layout(w, h, error_map);
		if (L.end > NOALLOC_SCRATCH_BYTES)
			throw InvalidArgument("frame exceeds the static scratch");
		unsigned char *base = nd.scratch;
		FrameDesc *frames = reinterpret_cast<FrameDesc *>(base + L.desc);
		FrameState *state = reinterpret_cast<FrameState *>(base + L.state);
		Control *ctl = reinterpret_cast<Control *>(base + L.ctl);
		long long *offsets = reinterpret_cast<long long *>(base + L.offsets);
		int2 *rows = reinterpret_cast<int2 *>(base + L.rows);
		int4 *items = reinterpret_cast<int4 *>(base + L.items);
		uint2 *targets = reinterpret_cast<uint2 *>(base + L.targets);
		uint2 *cands = reinterpret_cast<uint2 *>(base + L.cands);
		Seed *seeds = reinterpret_cast<Seed *>(base + L.seeds);

		FrameDesc fd{};
		fd.data = im->data;
		fd.error = im->error;
		fd.gain_map = im->error ? nullptr : im->gain;
		fd.rn_map = im->error ? nullptr : im->readnoise;
		fd.bg_map = im->background;
		fd.mask = im->mask;
		fd.clean = clean;
		fd.mask_out = mask;
		fd.bits = reinterpret_cast<uint32_t *>(base + L.bits);
		fd.gain = o->gain;
		fd.rn = o->readnoise;
		fd.bg = o->background;
		fd.w = w;
		fd.h = h;
		fd.words = (w + 31) / 32;
		fd.plane = L.plane;
		fd.pstride = L.plane;
		fd.has_bg = im->background != nullptr || !std::isnan(o->background);
		DetectParams prm{};
		prm.contrast = o->contrast;
		prm.cr = o->cr_threshold;
		prm.nb = o->neighbor_threshold;
		prm.tmin = std::fmin(o->cr_threshold, o->neighbor_threshold);
		prm.thi2 = 2 * o->cr_threshold * (1 - 1e-12);
		prm.tlo2 = 2 * o->neighbor_threshold * (1 - 1e-12);
		prm.mode = o->border;

		const int setup_n = h > L.nitems ? h : L.nitems;
		noalloc_setup_kernel<<<(setup_n + 255) / 256, 256, 0, s>>>(fd, frames, offsets, rows, items,
			L.nitems, error_map ? STREAM_ROWS : MTILE);
		init_kernel<<<1, 256, 0, s>>>(state, 1, ctl, o->maxiter,
			(unsigned long long)im->width * im->height);
		const int row_blocks = (h + 7) / 8 < nd.sms * 8 ? (h + 7) / 8 : nd.sms * 8;
		const int grow_items = (h + GROW_ROWS - 1) / GROW_ROWS * ((fd.words + 31) / 32);
		const int grow_blocks = (grow_items + 7) / 8 < nd.sms * 8 ? (grow_items + 7) / 8 : nd.sms * 8;
		if (!o->maxiter) {
			copy_kernel<<<row_blocks, 256, 0, s>>>(frames, rows, h);
		} else {
			// Bit planes start at zero (prepare_kernel writes HOLE, EXCL and
			// DONOR); the scratch keeps the previous call's contents.
			check(cudaMemsetAsync(fd.bits, 0, (size_t)N_PLANES * L.plane * sizeof(uint32_t), s));
			prepare_kernel<PREP_ANY><<<row_blocks, 256, 0, s>>>(frames, state, rows, h);
			fill_kernel<<<row_blocks, 256, 0, s>>>(frames, state, rows, h);
			for (int it = 0; it < o->maxiter; ++it) {
				if (error_map) {
					const int b = (L.nitems + 7) / 8 < nd.sms * 8 ? (L.nitems + 7) / 8 : nd.sms * 8;
					sig_stream_kernel<<<b, 256, 0, s>>>(frames, state, items, L.nitems, prm, ctl,
						cands);
				} else {
					const int b = L.nitems < nd.sms * 8 ? L.nitems : nd.sms * 8;
					sig_model_kernel<<<b, 256, 0, s>>>(frames, state, items, L.nitems, prm, ctl,
						cands);
				}
				// The dense kernels above zeroed S1, S2 and CAND.
				candidate_high_kernel<PATH_ANY><<<nd.sms * 8, 256, 0, s>>>(frames, cands, prm, ctl,
					seeds, 1);
				seed_kernel<<<nd.sms * 8, 256, 0, s>>>(frames, seeds, prm, ctl, 1);
				candidate_low_kernel<PATH_ANY><<<nd.sms * 8, 256, 0, s>>>(frames, cands, prm, ctl, 1);
				grow_kernel<<<grow_blocks, 256, 0, s>>>(frames, state, nullptr, grow_items, targets,
					ctl);
				control_kernel<<<1, 1024, 0, s>>>(state, 1, ctl, 0, 0);
				replace_kernel<<<nd.sms * 8, 256, 0, s>>>(frames, state, targets, &ctl->n_targets, nullptr,
					nullptr, nullptr);
			}
			restore_kernel<<<row_blocks, 256, 0, s>>>(frames, rows, h);
		}
		check(cudaGetLastError());
		FrameState st;
		check(cudaMemcpyAsync(&st, state, sizeof(st), cudaMemcpyDeviceToHost, s));
		check(cudaStreamSynchronize(s));
		check_state(st);
	}, msg, len);
}

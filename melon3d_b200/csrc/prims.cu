// Exclusive scan, stable LSD radix sort and key-range reduction; the launch
// accounting behind M3G_LAUNCH.
#include "prims.cuh"

#include <atomic>
#include <map>
#include <mutex>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <string>
#include <utility>
#include <vector>

namespace m3g
{

// ---- launch accounting --------------------------------------------------------

namespace
{
std::atomic<long long> gLaunches{ 0 };
std::mutex gMu;
std::string gTarget;
std::vector<cudaEvent_t> gPool;
struct TimedLaunch
{
	const char* name;
	cudaEvent_t start, stop;
};
std::vector<TimedLaunch> gPairs;
cudaEvent_t gOpen = nullptr;
double gTimedMs = 0.0;
long long gTimedLaunches = 0;
std::map<std::string, std::pair<double, long long>> gPerKernel; // "*" target: every kernel

// the selection: "*" (every kernel) or a comma-separated list of names
bool timed(const char* name)
{
	if (gTarget == "*")
	{
		return true;
	}
	const size_t len = strlen(name);
	size_t pos = 0;
	while (pos <= gTarget.size())
	{
		size_t end = gTarget.find(',', pos);
		end = end == std::string::npos ? gTarget.size() : end;
		if (end - pos == len && gTarget.compare(pos, len, name) == 0)
		{
			return true;
		}
		pos = end + 1;
	}
	return false;
}

cudaEvent_t takeEvent()
{
	if (!gPool.empty())
	{
		cudaEvent_t e = gPool.back();
		gPool.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	cudaEventCreate(&e);
	return e;
}

// fold finished event pairs into the running total (caller holds gMu)
void drainPairs()
{
	for (auto& p : gPairs)
	{
		float ms = 0.0f;
		cudaEventSynchronize(p.stop);
		cudaEventElapsedTime(&ms, p.start, p.stop);
		gTimedMs += ms;
		++gTimedLaunches;
		auto& k = gPerKernel[p.name];
		k.first += ms;
		++k.second;
		gPool.push_back(p.start);
		gPool.push_back(p.stop);
	}
	gPairs.clear();
}
} // namespace

namespace
{
std::atomic<long long> gH2D{ 0 }, gD2H{ 0 };
std::atomic<long long> gAllocations{ 0 };
}
void countAllocation() { gAllocations.fetch_add(1, std::memory_order_relaxed); }

cudaError_t countedMemcpyAsync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s)
{
	if (kind == cudaMemcpyHostToDevice)
	{
		gH2D.fetch_add((long long)bytes, std::memory_order_relaxed);
	}
	else if (kind == cudaMemcpyDeviceToHost)
	{
		gD2H.fetch_add((long long)bytes, std::memory_order_relaxed);
	}
	return (cudaMemcpyAsync)(dst, src, bytes, kind, s);
}

void launchBegin(const char* name, cudaStream_t s)
{
	gLaunches.fetch_add(1, std::memory_order_relaxed);
	if (gTarget.empty())
	{
		return;
	}
	std::lock_guard<std::mutex> lock(gMu);
	if (timed(name))
	{
		gOpen = takeEvent();
		cudaEventRecord(gOpen, s);
	}
}

void launchEnd(const char* name, cudaStream_t s)
{
	if (gTarget.empty())
	{
		return;
	}
	std::lock_guard<std::mutex> lock(gMu);
	if (gOpen != nullptr && timed(name))
	{
		cudaEvent_t stop = takeEvent();
		cudaEventRecord(stop, s);
		gPairs.push_back({ name, gOpen, stop });
		gOpen = nullptr;
		if (gPairs.size() >= 4096)
		{
			drainPairs();
		}
	}
}

// Test aid: with M3D_GPU_POISON_ALLOCATIONS=1 in the environment, every
// scratch buffer the library allocates starts filled with 0xA5 bytes instead
// of whatever the allocator hands back, so a kernel that reads memory it never
// wrote fails the same way on every run.
static bool poisonAllocations()
{
	static const bool on = [] {
		const char* v = getenv("M3D_GPU_POISON_ALLOCATIONS");
		return v != nullptr && v[0] == '1';
	}();
	return on;
}

bool DevBuf::ensure(size_t need)
{
	if (need <= bytes && ptr != nullptr)
	{
		return true;
	}
	size_t nb = bytes * 2 > need ? bytes * 2 : need;
	if (nb < 256)
	{
		nb = 256;
	}
	void* p = nullptr;
	if (cudaMalloc(&p, nb) != cudaSuccess)
	{
		return false;
	}
	countAllocation();
	if (poisonAllocations())
	{
		// the fill runs on the legacy stream, which the worlds' non-blocking
		// streams do not wait for: finish it before anything uses the buffer
		cudaMemset(p, 0xA5, nb);
		cudaDeviceSynchronize();
	}
	if (ptr != nullptr)
	{
		cudaFree(ptr);
	}
	ptr = p;
	bytes = nb;
	return true;
}

bool DevBuf::ensureZeroed(size_t need, cudaStream_t stream)
{
	void* before = ptr;
	if (!ensure(need))
	{
		return false;
	}
	if (ptr != before)
	{
		cudaMemsetAsync(ptr, 0, bytes, stream);
	}
	return true;
}

void DevBuf::release()
{
	if (ptr != nullptr)
	{
		cudaFree(ptr);
	}
	ptr = nullptr;
	bytes = 0;
}

void PrimScratch::release()
{
	scanStatus.release();
	scanTicket.release();
	waitError.release();
	sortKeys.release();
	sortVals.release();
	sortCounts.release();
	sortOffs.release();
	scanIn.release();
	reduce.release();
	if (hostReduce != nullptr)
	{
		cudaFreeHost(hostReduce);
		hostReduce = nullptr;
	}
}

// ---------------------------------------------------------------------------
// scan: one pass with decoupled look-back.  Each CTA takes the next 2048-word
// tile from a ticket counter (so a CTA only ever waits on tiles whose CTAs
// are already running), publishes its tile total, then its warp 0 walks back
// over the predecessors' published words, 32 at a time, until it meets an
// inclusive prefix.  Status words carry the call's epoch, so words left by
// earlier calls read as "not yet published" and nothing is cleared between
// calls.  Waits are bounded: a wait that runs out counts as a zero
// contribution and raises the caller's error word.
// ---------------------------------------------------------------------------

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr uint32_t kLookbackSpinLimit = 1u << 22;
constexpr uint32_t kEpochLimit = 1u << 30;

__device__ __forceinline__ uint32_t warpInclusive(uint32_t v)
{
	int lane = threadIdx.x & 31;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1)
	{
		uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
		if (lane >= o)
		{
			v += t;
		}
	}
	return v;
}

__device__ __forceinline__ uint32_t warpSum(uint32_t v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
	{
		v += __shfl_xor_sync(0xffffffffu, v, o);
	}
	return v;
}

// exclusive scan of one value per thread across the CTA; the CTA total is
// left in warpSums[kScanThreads / 32]
__device__ uint32_t blockExclusive(uint32_t v, uint32_t* warpSums)
{
	int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	uint32_t inc = warpInclusive(v);
	if (lane == 31)
	{
		warpSums[warp] = inc;
	}
	__syncthreads();
	if (warp == 0)
	{
		uint32_t ws = lane < (kScanThreads / 32) ? warpSums[lane] : 0u;
		uint32_t wi = warpInclusive(ws);
		if (lane < (kScanThreads / 32))
		{
			warpSums[lane] = wi - ws;
		}
		if (lane == (kScanThreads / 32) - 1)
		{
			warpSums[kScanThreads / 32] = wi;
		}
	}
	__syncthreads();
	uint32_t r = inc - v + warpSums[warp];
	return r;
}

// status word: epoch (30 bits) << 34 | flag (1 aggregate, 2 inclusive) << 32 | value
__device__ __forceinline__ uint64_t statusWord(uint32_t epoch, uint32_t flag, uint32_t value)
{
	return ((uint64_t)epoch << 34) | ((uint64_t)flag << 32) | value;
}

// One launch scans one or two independent arrays (segments): segment 1's
// tiles follow segment 0's in the ticket order and look back only as far as
// its own first tile.
struct ScanSeg
{
	const uint32_t* in;
	uint32_t* out;
	int64_t n;
	uint32_t* total;
	int32_t tile0, tiles;
};
struct ScanSegs
{
	ScanSeg s[2];
	int32_t count, allTiles;
};

// Decoupled look-back scan.  A tile's wait for a predecessor's status is
// bounded (spinLimit unsuccessful polls; 0: the tile does not wait at all).
// A tile that gives up raises the error word and computes its prefix by
// summing the inputs of all earlier tiles directly: slower, but the same
// exact result, so no later kernel ever indexes with a partial prefix.
__global__ void __launch_bounds__(kScanThreads)
	kScanLookback(ScanSegs segs, uint64_t* status, uint32_t* ticket, uint32_t epoch, uint32_t* error,
				  int64_t spinLimit)
{
	M3G_KERNEL_BEGIN();
	__shared__ uint32_t warpSums[kScanThreads / 32 + 1];
	__shared__ uint32_t sTile, sPrefix;
	if (threadIdx.x == 0)
	{
		sTile = atomicAdd(&ticket[0], 1u);
	}
	__syncthreads();
	const int t = (int)sTile; // global tile: status word index
	const bool second = segs.count > 1 && t >= segs.s[1].tile0;
	const uint32_t* in = second ? segs.s[1].in : segs.s[0].in;
	uint32_t* out = second ? segs.s[1].out : segs.s[0].out;
	const int64_t n = second ? segs.s[1].n : segs.s[0].n;
	uint32_t* total = second ? segs.s[1].total : segs.s[0].total;
	const int first = second ? segs.s[1].tile0 : 0; // the segment's first global tile
	const int tiles = second ? segs.s[1].tiles : segs.s[0].tiles;
	const int lt = t - first; // tile inside the segment
	const int64_t base = (int64_t)lt * kScanTile + (int64_t)threadIdx.x * kScanItems;
	uint32_t vals[kScanItems];
	uint32_t sum = 0;
#pragma unroll
	for (int k = 0; k < kScanItems; ++k)
	{
		int64_t i = base + k;
		vals[k] = i < n ? in[i] : 0u;
		sum += vals[k];
	}
	uint32_t pre = blockExclusive(sum, warpSums);
	const uint32_t agg = warpSums[kScanThreads / 32];
	volatile uint64_t* vs = status;
	if (threadIdx.x < 32)
	{
		const int lane = threadIdx.x;
		uint32_t excl = 0;
		if (lt == 0)
		{
			if (lane == 0)
			{
				vs[t] = statusWord(epoch, 2u, agg);
			}
		}
		else
		{
			if (lane == 0)
			{
				vs[t] = statusWord(epoch, 1u, agg);
			}
			int idx = t - 1;
			bool fallback = false;
			while (true)
			{
				const int j = idx - lane;
				uint32_t flag = 2u, value = 0u; // lanes before the segment's first tile contribute nothing
				bool gaveUp = false;
				if (j >= first)
				{
					flag = 0u;
					for (int64_t it = 0; flag == 0u; ++it)
					{
						if (it >= spinLimit)
						{
							gaveUp = true;
							flag = 2u;
							break;
						}
						uint64_t w = vs[j];
						if ((uint32_t)(w >> 34) == epoch)
						{
							flag = (uint32_t)(w >> 32) & 3u;
							value = (uint32_t)w;
						}
					}
				}
				if (__any_sync(0xffffffffu, gaveUp))
				{
					fallback = true;
					break;
				}
				const uint32_t inclusive = __ballot_sync(0xffffffffu, flag == 2u);
				if (inclusive != 0u)
				{
					const int stop = __ffs((int)inclusive) - 1;
					excl += warpSum(lane <= stop ? value : 0u);
					break;
				}
				excl += warpSum(value);
				idx -= 32;
			}
			if (fallback)
			{
				if (lane == 0)
				{
					atomicOr(error, 1u);
				}
				uint32_t s = 0;
				const int64_t end = (int64_t)lt * kScanTile;
				for (int64_t i = lane; i < end; i += 32)
				{
					s += in[i];
				}
				excl = warpSum(s);
			}
			if (lane == 0)
			{
				vs[t] = statusWord(epoch, 2u, excl + agg);
			}
		}
		if (lane == 0)
		{
			sPrefix = excl;
		}
	}
	__syncthreads();
	pre += sPrefix;
#pragma unroll
	for (int k = 0; k < kScanItems; ++k)
	{
		int64_t i = base + k;
		if (i < n)
		{
			out[i] = pre;
		}
		pre += vals[k];
	}
	if (threadIdx.x == 0)
	{
		if (lt == tiles - 1 && total != nullptr)
		{
			*total = sPrefix + agg;
		}
		// the last CTA to finish rewinds the ticket for the next call
		if (atomicAdd(&ticket[1], 1u) == (uint32_t)segs.allTiles - 1u)
		{
			ticket[0] = 0u;
			ticket[1] = 0u;
		}
	}
}

// Copy an in-place multi-tile scan's input aside (a tile that gives up
// re-reads the inputs of the tiles before it).
static const uint32_t* scanInput(const uint32_t* in, uint32_t* out, int64_t n, PrimScratch& s, cudaStream_t stream)
{
	if (in == out && n > kScanTile)
	{
		s.scanIn.ensure((size_t)n * sizeof(uint32_t));
		cudaMemcpyAsync(s.scanIn.ptr, in, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream);
		return s.scanIn.as<uint32_t>();
	}
	return in;
}

static void launchScan(ScanSegs& g, PrimScratch& s, cudaStream_t stream)
{
	s.scanTicket.ensureZeroed(4 * sizeof(uint32_t), stream);
	s.waitError.ensureZeroed(4 * sizeof(uint32_t), stream);
	void* before = s.scanStatus.ptr;
	s.scanStatus.ensureZeroed((size_t)(g.allTiles + 1) * sizeof(uint64_t), stream);
	if (s.scanStatus.ptr != before || ++s.scanEpoch >= kEpochLimit)
	{
		// fresh (zeroed) status words, or the epoch wrapped: restart at 1
		if (s.scanStatus.ptr == before)
		{
			cudaMemsetAsync(s.scanStatus.ptr, 0, s.scanStatus.bytes, stream);
		}
		s.scanEpoch = 1;
	}
	uint32_t* err = s.errorWord != nullptr ? s.errorWord : s.waitError.as<uint32_t>();
	M3G_LAUNCH(kScanLookback, (unsigned)g.allTiles, kScanThreads, stream, g, s.scanStatus.as<uint64_t>(),
			   s.scanTicket.as<uint32_t>(), s.scanEpoch, err,
			   s.waitLimit >= 0 ? s.waitLimit : (int64_t)kLookbackSpinLimit);
}

void scanExclusive(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total, PrimScratch& s,
				   cudaStream_t stream)
{
	if (n <= 0)
	{
		if (total != nullptr)
		{
			fillWords(total, 0u, sizeof(uint32_t), stream);
		}
		return;
	}
	ScanSegs g = {};
	g.s[0] = { scanInput(in, out, n, s, stream), out, n, total, 0, (int32_t)((n + kScanTile - 1) / kScanTile) };
	g.count = 1;
	g.allTiles = g.s[0].tiles;
	launchScan(g, s, stream);
}

void scanExclusive2(const uint32_t* in0, uint32_t* out0, int64_t n0, uint32_t* total0, const uint32_t* in1,
					uint32_t* out1, int64_t n1, uint32_t* total1, PrimScratch& s, cudaStream_t stream)
{
	if (n0 <= 0 || n1 <= 0 || in0 == out0 || in1 == out1)
	{
		scanExclusive(in0, out0, n0, total0, s, stream);
		scanExclusive(in1, out1, n1, total1, s, stream);
		return;
	}
	ScanSegs g = {};
	const int32_t t0 = (int32_t)((n0 + kScanTile - 1) / kScanTile);
	const int32_t t1 = (int32_t)((n1 + kScanTile - 1) / kScanTile);
	g.s[0] = { in0, out0, n0, total0, 0, t0 };
	g.s[1] = { in1, out1, n1, total1, t0, t1 };
	g.count = 2;
	g.allTiles = t0 + t1;
	launchScan(g, s, stream);
}

// ---------------------------------------------------------------------------
// radix sort: 8-bit digits, 256 threads x 8 items per tile, warp-contiguous
// item ownership so the tile order equals the input order (stability)
// ---------------------------------------------------------------------------

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadix = 256;

__device__ __forceinline__ int64_t effectiveN(int64_t nMax, const uint32_t* nDev)
{
	if (nDev == nullptr)
	{
		return nMax;
	}
	int64_t d = (int64_t)*nDev;
	return d < nMax ? d : nMax;
}

__global__ void kSortHistogram(const uint64_t* keys, int64_t nMax, const uint32_t* nDev, int shift, uint64_t bias,
							   uint32_t* counts, int tiles)
{
	M3G_KERNEL_BEGIN();
	__shared__ uint32_t hist[kRadix];
	const int64_t n = effectiveN(nMax, nDev);
	for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
	{
		hist[d] = 0;
	}
	__syncthreads();
	int64_t base = (int64_t)blockIdx.x * kSortTile;
	for (int k = threadIdx.x; k < kSortTile; k += kSortThreads)
	{
		int64_t i = base + k;
		if (i < n)
		{
			atomicAdd(&hist[(uint32_t)((keys[i] - bias) >> shift) & 0xFFu], 1u);
		}
	}
	__syncthreads();
	for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
	{
		counts[(int64_t)d * tiles + blockIdx.x] = hist[d];
	}
}

__global__ void kSortScatter(const uint64_t* keysIn, const uint32_t* valsIn, uint64_t* keysOut, uint32_t* valsOut,
							 int64_t nMax, const uint32_t* nDev, int shift, uint64_t bias, const uint32_t* offsets,
							 int tiles)
{
	M3G_KERNEL_BEGIN();
	__shared__ uint32_t warpHist[kSortWarps][kRadix];
	const int64_t n = effectiveN(nMax, nDev);
	int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int d = threadIdx.x; d < kSortWarps * kRadix; d += kSortThreads)
	{
		(&warpHist[0][0])[d] = 0;
	}
	__syncthreads();
	int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * (32 * kSortItems);
	uint32_t lt = (1u << lane) - 1u;

	// pass 1: per-warp digit counts
	for (int r = 0; r < kSortItems; ++r)
	{
		int64_t i = base + r * 32 + lane;
		bool valid = i < n;
		uint32_t d = valid ? ((uint32_t)((keysIn[i] - bias) >> shift) & 0xFFu) : 0x100u;
		uint32_t peers = __match_any_sync(0xffffffffu, d);
		if (valid && (peers & lt) == 0)
		{
			warpHist[warp][d] += __popc(peers);
		}
		__syncwarp();
	}
	__syncthreads();
	// exclusive prefix over warps, plus the tile's global digit base
	for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
	{
		uint32_t run = offsets[(int64_t)d * tiles + blockIdx.x];
		for (int w = 0; w < kSortWarps; ++w)
		{
			uint32_t c = warpHist[w][d];
			warpHist[w][d] = run;
			run += c;
		}
	}
	__syncthreads();
	// pass 2: stable ranks and scatter
	for (int r = 0; r < kSortItems; ++r)
	{
		int64_t i = base + r * 32 + lane;
		bool valid = i < n;
		uint64_t key = valid ? keysIn[i] : 0ull;
		uint32_t d = valid ? ((uint32_t)((key - bias) >> shift) & 0xFFu) : 0x100u;
		uint32_t peers = __match_any_sync(0xffffffffu, d);
		if (valid)
		{
			uint32_t pos = warpHist[warp][d] + __popc(peers & lt);
			keysOut[pos] = key;
			valsOut[pos] = valsIn[i];
		}
		__syncwarp();
		if (valid && (peers & lt) == 0)
		{
			warpHist[warp][d] += __popc(peers);
		}
		__syncwarp();
	}
}

__global__ void kCopyPairs(const uint64_t* ks, const uint32_t* vs, uint64_t* kd, uint32_t* vd, int64_t nMax,
						   const uint32_t* nDev)
{
	M3G_KERNEL_BEGIN();
	const int64_t n = effectiveN(nMax, nDev);
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		kd[i] = ks[i];
		vd[i] = vs[i];
	}
}

void radixSortPairs(uint64_t* keys, uint32_t* vals, int64_t n, uint64_t varyMask, PrimScratch& s,
					cudaStream_t stream, const uint32_t* nDev, uint64_t bias)
{
	if (n <= 1)
	{
		return;
	}
	int tiles = (int)((n + kSortTile - 1) / kSortTile);
	s.sortKeys.ensure((size_t)n * sizeof(uint64_t));
	s.sortVals.ensure((size_t)n * sizeof(uint32_t));
	s.sortCounts.ensure((size_t)kRadix * tiles * sizeof(uint32_t));
	s.sortOffs.ensure((size_t)kRadix * tiles * sizeof(uint32_t));
	uint64_t* k0 = keys;
	uint32_t* v0 = vals;
	uint64_t* k1 = s.sortKeys.as<uint64_t>();
	uint32_t* v1 = s.sortVals.as<uint32_t>();
	uint32_t* counts = s.sortCounts.as<uint32_t>();
	uint32_t* offs = s.sortOffs.as<uint32_t>();
	// 8-bit digit windows placed greedily on the bits that vary among the keys
	// (constant bits need no pass): each window starts at the lowest varying
	// bit not yet covered, clamped so it stays inside the key.  Windows rise
	// monotonically, which keeps the LSD sort exact even where two overlap.
	int passes = 0;
	uint64_t remaining = varyMask;
	while (remaining != 0)
	{
		int shift = __builtin_ctzll(remaining);
		shift = shift > 56 ? 56 : shift;
		remaining &= ~(0xFFull << shift);
		M3G_LAUNCH(kSortHistogram, tiles, kSortThreads, stream, k0, n, nDev, shift, bias, counts, tiles);
		scanExclusive(counts, offs, (int64_t)kRadix * tiles, nullptr, s, stream);
		M3G_LAUNCH(kSortScatter, tiles, kSortThreads, stream, k0, v0, k1, v1, n, nDev, shift, bias, offs, tiles);
		uint64_t* tk = k0;
		k0 = k1;
		k1 = tk;
		uint32_t* tv = v0;
		v0 = v1;
		v1 = tv;
		++passes;
	}
	if (passes & 1)
	{
		M3G_LAUNCH(kCopyPairs, blocksFor(n, 256), 256, stream, k0, v0, keys, vals, n, nDev);
	}
}

__global__ void kReduceInit(uint64_t* r)
{
	M3G_KERNEL_BEGIN();
	r[0] = 0ull;
	r[1] = ~0ull;
}

__global__ void kReduceKeys(const uint64_t* keys, int64_t n, uint64_t* r)
{
	M3G_KERNEL_BEGIN();
	uint64_t o = 0ull, a = ~0ull;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
	{
		uint64_t k = keys[i];
		o |= k;
		a &= k;
	}
	for (int off = 16; off > 0; off >>= 1)
	{
		o |= __shfl_xor_sync(0xffffffffu, o, off);
		a &= __shfl_xor_sync(0xffffffffu, a, off);
	}
	if ((threadIdx.x & 31) == 0)
	{
		atomicOr((unsigned long long*)&r[0], (unsigned long long)o);
		atomicAnd((unsigned long long*)&r[1], (unsigned long long)a);
	}
}

__device__ __forceinline__ void fillRange(uint32_t* p, uint32_t v, int64_t words, int64_t i, int64_t stride)
{
	if (((uintptr_t)p & 15u) == 0 && (words & 3) == 0)
	{
		uint4* q = (uint4*)p;
		const uint4 v4 = make_uint4(v, v, v, v);
		for (; i < words / 4; i += stride)
		{
			q[i] = v4;
		}
		return;
	}
	for (; i < words; i += stride)
	{
		p[i] = v;
	}
}

// one or two ranges (p1 null: one)
__global__ void kFillWords(uint32_t* p0, uint32_t v0, int64_t words0, uint32_t* p1, uint32_t v1, int64_t words1)
{
	M3G_KERNEL_BEGIN();
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	fillRange(p0, v0, words0, i, stride);
	if (p1 != nullptr)
	{
		fillRange(p1, v1, words1, i, stride);
	}
}

static int fillBlocks(int64_t words)
{
	int blocks = blocksFor(words, 256 * 4);
	return blocks > 4 * 148 ? 4 * 148 : blocks;
}

void fillWords(void* p, uint32_t v, size_t bytes, cudaStream_t stream)
{
	const int64_t words = (int64_t)(bytes / sizeof(uint32_t));
	if (words <= 0)
	{
		return;
	}
	M3G_LAUNCH(kFillWords, fillBlocks(words), 256, stream, (uint32_t*)p, v, words, (uint32_t*)nullptr, 0u,
			   (int64_t)0);
}

void fillWords2(void* p0, uint32_t v0, size_t bytes0, void* p1, uint32_t v1, size_t bytes1, cudaStream_t stream)
{
	const int64_t w0 = (int64_t)(bytes0 / sizeof(uint32_t)), w1 = (int64_t)(bytes1 / sizeof(uint32_t));
	if (w0 <= 0 || w1 <= 0)
	{
		fillWords(p0, v0, bytes0, stream);
		fillWords(p1, v1, bytes1, stream);
		return;
	}
	M3G_LAUNCH(kFillWords, fillBlocks(w0 > w1 ? w0 : w1), 256, stream, (uint32_t*)p0, v0, w0, (uint32_t*)p1, v1, w1);
}

void reduceKeyRange(const uint64_t* keys, int64_t n, PrimScratch& s, cudaStream_t stream)
{
	s.reduce.ensure(2 * sizeof(uint64_t));
	if (s.hostReduce == nullptr)
	{
		cudaMallocHost((void**)&s.hostReduce, 2 * sizeof(uint64_t));
	}
	M3G_LAUNCH(kReduceInit, 1, 1, stream, s.reduce.as<uint64_t>());
	if (n > 0)
	{
		int blocks = blocksFor(n, 256);
		blocks = blocks > 1184 ? 1184 : blocks;
		M3G_LAUNCH(kReduceKeys, blocks, 256, stream, keys, n, s.reduce.as<uint64_t>());
	}
	cudaMemcpyAsync(s.hostReduce, s.reduce.ptr, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream);
}

} // namespace m3g

extern "C"
{

// Select the kernel to time ("" or NULL: none; "*": every kernel) and zero
// the counters.
void m3d_gpu_profiler_reset(const char* kernelName)
{
	std::lock_guard<std::mutex> lock(m3g::gMu);
	m3g::drainPairs();
	m3g::gTarget = kernelName != nullptr ? kernelName : "";
	m3g::gTimedMs = 0.0;
	m3g::gTimedLaunches = 0;
	m3g::gPerKernel.clear();
	m3g::gOpen = nullptr;
	m3g::gLaunches.store(0);
	m3g::gH2D.store(0);
	m3g::gD2H.store(0);
}

// Host->device and device->host bytes copied by the library since the last reset.
void m3d_gpu_profiler_bytes(long long* h2d, long long* d2h)
{
	if (h2d != nullptr)
	{
		*h2d = m3g::gH2D.load();
	}
	if (d2h != nullptr)
	{
		*d2h = m3g::gD2H.load();
	}
}

// Kernel launches of the library since the last reset (all kernels).
long long m3d_gpu_profiler_launches(void) { return m3g::gLaunches.load(); }

// Device allocations (cudaMalloc) the library made since it was loaded.
long long m3d_gpu_profiler_allocations(void) { return m3g::gAllocations.load(); }

// Total device time (ms) and launch count of the selected kernel since the
// last reset, from CUDA events recorded around each of its launches.
void m3d_gpu_profiler_kernel(float* totalMs, int32_t* launches)
{
	std::lock_guard<std::mutex> lock(m3g::gMu);
	m3g::drainPairs();
	if (totalMs != nullptr)
	{
		*totalMs = (float)m3g::gTimedMs;
	}
	if (launches != nullptr)
	{
		*launches = (int32_t)m3g::gTimedLaunches;
	}
}

// Per-kernel table of the timed launches since the last reset, one line per
// kernel: "<name> <launches> <total ms>\n".  Returns the length of the whole
// table; writes at most capacity-1 characters and a terminating NUL.
int32_t m3d_gpu_profiler_table(char* out, int32_t capacity)
{
	std::lock_guard<std::mutex> lock(m3g::gMu);
	m3g::drainPairs();
	std::string t;
	char line[160];
	for (const auto& k : m3g::gPerKernel)
	{
		snprintf(line, sizeof(line), "%s %lld %.6f\n", k.first.c_str(), k.second.second, k.second.first);
		t += line;
	}
	if (out != nullptr && capacity > 0)
	{
		size_t n = t.size() < (size_t)capacity - 1 ? t.size() : (size_t)capacity - 1;
		memcpy(out, t.data(), n);
		out[n] = 0;
	}
	return (int32_t)t.size();
}

} // extern "C"

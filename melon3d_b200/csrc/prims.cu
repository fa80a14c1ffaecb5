// Exclusive scan, stable LSD radix sort and key-range reduction; the launch
// accounting behind M3G_LAUNCH.
#include "prims.cuh"

#include <atomic>
#include <mutex>
#include <stdio.h>
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
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> gPairs;
cudaEvent_t gOpen = nullptr;
double gTimedMs = 0.0;
long long gTimedLaunches = 0;

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
		cudaEventSynchronize(p.second);
		cudaEventElapsedTime(&ms, p.first, p.second);
		gTimedMs += ms;
		++gTimedLaunches;
		gPool.push_back(p.first);
		gPool.push_back(p.second);
	}
	gPairs.clear();
}
} // namespace

namespace
{
std::atomic<long long> gH2D{ 0 }, gD2H{ 0 };
}

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
	if (gTarget == name)
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
	if (gOpen != nullptr && gTarget == name)
	{
		cudaEvent_t stop = takeEvent();
		cudaEventRecord(stop, s);
		gPairs.emplace_back(gOpen, stop);
		gOpen = nullptr;
		if (gPairs.size() >= 4096)
		{
			drainPairs();
		}
	}
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
	scanA.release();
	scanB.release();
	scanC.release();
	sortKeys.release();
	sortVals.release();
	sortCounts.release();
	reduce.release();
	if (hostReduce != nullptr)
	{
		cudaFreeHost(hostReduce);
		hostReduce = nullptr;
	}
}

// ---------------------------------------------------------------------------
// scan: 256 threads x 8 items per block; block totals are scanned recursively
// ---------------------------------------------------------------------------

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

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

// exclusive scan of one tile in place; returns the tile total to thread 0..N
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

__global__ void kScanTiles(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* tileSums)
{
	__shared__ uint32_t warpSums[kScanThreads / 32 + 1];
	int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
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
	if (threadIdx.x == 0 && tileSums != nullptr)
	{
		tileSums[blockIdx.x] = warpSums[kScanThreads / 32];
	}
}

__global__ void kScanAdd(uint32_t* out, int64_t n, const uint32_t* tileOffsets)
{
	int64_t base = (int64_t)blockIdx.x * kScanTile;
	uint32_t add = tileOffsets[blockIdx.x];
	for (int k = threadIdx.x; k < kScanTile; k += kScanThreads)
	{
		int64_t i = base + k;
		if (i < n)
		{
			out[i] += add;
		}
	}
}

__global__ void kScanTotal(const uint32_t* in, const uint32_t* out, int64_t n, uint32_t* total)
{
	*total = n > 0 ? out[n - 1] + in[n - 1] : 0u;
}

// total of a single-tile scan is produced by kScanTiles into tileSums
static void scanLevel(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total, DevBuf* levels, int level,
					  cudaStream_t stream)
{
	int64_t tiles = (n + kScanTile - 1) / kScanTile;
	if (tiles <= 1)
	{
		M3G_LAUNCH(kScanTiles, 1, kScanThreads, stream, in, out, n, total);
		return;
	}
	levels[level].ensure((size_t)tiles * sizeof(uint32_t));
	uint32_t* sums = levels[level].as<uint32_t>();
	M3G_LAUNCH(kScanTiles, (unsigned)tiles, kScanThreads, stream, in, out, n, sums);
	scanLevel(sums, sums, tiles, total, levels, level + 1, stream);
	M3G_LAUNCH(kScanAdd, (unsigned)tiles, kScanThreads, stream, out, n, sums);
}

void scanExclusive(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total, PrimScratch& s,
				   cudaStream_t stream)
{
	if (n <= 0)
	{
		if (total != nullptr)
		{
			cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
		}
		return;
	}
	DevBuf levels[3] = {};
	levels[0] = s.scanA;
	levels[1] = s.scanB;
	levels[2] = s.scanC;
	// the in-place aliasing is fine: each tile reads all its inputs before
	// writing, and tiles are disjoint
	if (total == nullptr)
	{
		// scan the tile sums without a total: reuse a scratch word
		levels[2].ensure(sizeof(uint32_t) * 4);
	}
	uint32_t* tot = total != nullptr ? total : levels[2].as<uint32_t>();
	scanLevel(in, out, n, tot, levels, 0, stream);
	s.scanA = levels[0];
	s.scanB = levels[1];
	s.scanC = levels[2];
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

__global__ void kSortHistogram(const uint64_t* keys, int64_t nMax, const uint32_t* nDev, int shift, uint32_t* counts,
							   int tiles)
{
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
			atomicAdd(&hist[(uint32_t)(keys[i] >> shift) & 0xFFu], 1u);
		}
	}
	__syncthreads();
	for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
	{
		counts[(int64_t)d * tiles + blockIdx.x] = hist[d];
	}
}

__global__ void kSortScatter(const uint64_t* keysIn, const uint32_t* valsIn, uint64_t* keysOut, uint32_t* valsOut,
							 int64_t nMax, const uint32_t* nDev, int shift, const uint32_t* offsets, int tiles)
{
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
		uint32_t d = valid ? ((uint32_t)(keysIn[i] >> shift) & 0xFFu) : 0x100u;
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
		uint32_t d = valid ? ((uint32_t)(key >> shift) & 0xFFu) : 0x100u;
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
	const int64_t n = effectiveN(nMax, nDev);
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		kd[i] = ks[i];
		vd[i] = vs[i];
	}
}

void radixSortPairs(uint64_t* keys, uint32_t* vals, int64_t n, uint64_t varyMask, PrimScratch& s,
					cudaStream_t stream, const uint32_t* nDev)
{
	if (n <= 1)
	{
		return;
	}
	int tiles = (int)((n + kSortTile - 1) / kSortTile);
	s.sortKeys.ensure((size_t)n * sizeof(uint64_t));
	s.sortVals.ensure((size_t)n * sizeof(uint32_t));
	s.sortCounts.ensure((size_t)kRadix * tiles * sizeof(uint32_t));
	uint64_t* k0 = keys;
	uint32_t* v0 = vals;
	uint64_t* k1 = s.sortKeys.as<uint64_t>();
	uint32_t* v1 = s.sortVals.as<uint32_t>();
	uint32_t* counts = s.sortCounts.as<uint32_t>();
	int passes = 0;
	for (int shift = 0; shift < 64; shift += 8)
	{
		if (((varyMask >> shift) & 0xFFull) == 0)
		{
			continue;
		}
		M3G_LAUNCH(kSortHistogram, tiles, kSortThreads, stream, k0, n, nDev, shift, counts, tiles);
		scanExclusive(counts, counts, (int64_t)kRadix * tiles, nullptr, s, stream);
		M3G_LAUNCH(kSortScatter, tiles, kSortThreads, stream, k0, v0, k1, v1, n, nDev, shift, counts, tiles);
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
	r[0] = 0ull;
	r[1] = ~0ull;
}

__global__ void kReduceKeys(const uint64_t* keys, int64_t n, uint64_t* r)
{
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

// Select the kernel to time ("" or NULL: none) and zero the counters.
void m3d_gpu_profiler_reset(const char* kernelName)
{
	std::lock_guard<std::mutex> lock(m3g::gMu);
	m3g::drainPairs();
	m3g::gTarget = kernelName != nullptr ? kernelName : "";
	m3g::gTimedMs = 0.0;
	m3g::gTimedLaunches = 0;
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

} // extern "C"

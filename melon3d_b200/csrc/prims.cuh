// Data-parallel building blocks used by the step: exclusive scan, stable
// LSD radix sort of (u64 key, u32 value) pairs, key-range reduction and an
// open-addressing set of 64-bit pair keys.  All hand-written for sm_100a;
// no library sort or scan is used on the stepping path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace m3g
{

// Grow-only device buffer, freed with its owner.
struct DevBuf
{
	void* ptr = nullptr;
	size_t bytes = 0;
	DevBuf() = default;
	DevBuf(const DevBuf&) = delete;
	DevBuf& operator=(const DevBuf&) = delete;
	~DevBuf() { release(); }
	bool ensure(size_t need);
	// like ensure(), but a fresh allocation is zero-filled on `stream`
	bool ensureZeroed(size_t need, cudaStream_t stream);
	void release();
	template <typename T>
	T* as() const
	{
		return (T*)ptr;
	}
};

// Scratch owned by the caller of the primitives.
struct PrimScratch
{
	DevBuf scanStatus;           // u64 per scan tile: epoch | flag | value
	DevBuf scanTicket;           // tile ticket + finished-CTA count (rewound by each scan)
	uint32_t scanEpoch = 0;      // epoch of the last scan launched
	DevBuf waitError;            // fallback error word when errorWord is not set
	uint32_t* errorWord = nullptr; // device word raised when a bounded wait runs out
	int64_t waitLimit = -1;        // polls before a wait gives up; < 0: the default
	DevBuf sortKeys, sortVals;   // ping-pong partner of a radix sort
	DevBuf sortCounts;           // per-tile digit histograms
	DevBuf sortOffs;             // their exclusive scan (the scatter's offsets)
	DevBuf scanIn;               // copy of the input of an in-place scan
	DevBuf reduce;               // 2 x u64: OR and AND of the keys
	DevBuf hostPinned;           // not device memory: see hostReduce
	uint64_t* hostReduce = nullptr; // pinned host copy of the reduce words
	void release();
};

// out[i] = sum(in[0..i)) for i < n; *total = sum(in[0..n)) when total != null.
// A tile whose look-back gives up re-reads the inputs of the earlier tiles, so
// an in-place scan (out == in) first copies its input aside.
// in and out may alias.
void scanExclusive(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total, PrimScratch& s,
				   cudaStream_t stream);
// Two independent scans (different arrays, neither in place) in one launch,
// with the results of two scanExclusive calls.
void scanExclusive2(const uint32_t* in0, uint32_t* out0, int64_t n0, uint32_t* total0, const uint32_t* in1,
					uint32_t* out1, int64_t n1, uint32_t* total1, PrimScratch& s, cudaStream_t stream);

// Stable sort of n (key, val) pairs by key.  Digits are taken from
// (key - bias), which must preserve the key order over the keys sorted (every
// key >= bias field by field, no borrows); only the bits of (key - bias) in
// `varyMask` are examined, by 8-bit windows placed on them.  When nDev is
// given, the element count is min(n, *nDev) read on the device (n is then the
// host-side upper bound that sizes the grid).  Result lands back in
// keys/vals, with the original keys.
void radixSortPairs(uint64_t* keys, uint32_t* vals, int64_t n, uint64_t varyMask, PrimScratch& s,
					cudaStream_t stream, const uint32_t* nDev = nullptr, uint64_t bias = 0ull);

// p[0 .. bytes/4) = v, as a kernel of the library (a memset node would break
// the stream's programmatic launch chain); bytes must be a multiple of 4.
void fillWords(void* p, uint32_t v, size_t bytes, cudaStream_t stream);
// two such fills in one launch
void fillWords2(void* p0, uint32_t v0, size_t bytes0, void* p1, uint32_t v1, size_t bytes1, cudaStream_t stream);

// Device-side OR / AND of n keys into s.reduce (two u64 words), then copied
// to the pinned host words s.hostReduce[0..1] (stream-ordered, no sync).
void reduceKeyRange(const uint64_t* keys, int64_t n, PrimScratch& s, cudaStream_t stream);

// Keys of an open-addressing hash set: 0xFFFF...F marks an empty slot.
constexpr uint64_t kEmptyKey = ~0ull;

__device__ __forceinline__ uint32_t hashKey(uint64_t k)
{
	k ^= k >> 33;
	k *= 0xff51afd7ed558ccdull;
	k ^= k >> 33;
	k *= 0xc4ceb9fe1a85ec53ull;
	k ^= k >> 33;
	return (uint32_t)k;
}

// insert; returns the slot index holding the key (capacity is a power of two)
__device__ __forceinline__ uint32_t hashInsert(uint64_t* table, uint32_t capMask, uint64_t key)
{
	uint32_t slot = hashKey(key) & capMask;
	for (uint32_t probe = 0; probe <= capMask; ++probe)
	{
		unsigned long long prev = atomicCAS((unsigned long long*)&table[slot], (unsigned long long)kEmptyKey,
											(unsigned long long)key);
		if (prev == kEmptyKey || prev == key)
		{
			return slot;
		}
		slot = (slot + 1) & capMask;
	}
	return 0xFFFFFFFFu; // full (the caller sizes the table to at least 2x the keys)
}

__device__ __forceinline__ bool hashContains(const uint64_t* table, uint32_t capMask, uint64_t key)
{
	uint32_t slot = hashKey(key) & capMask;
	for (uint32_t probe = 0; probe <= capMask; ++probe)
	{
		uint64_t k = table[slot];
		if (k == key)
		{
			return true;
		}
		if (k == kEmptyKey)
		{
			return false;
		}
		slot = (slot + 1) & capMask;
	}
	return false;
}

inline int blocksFor(int64_t n, int threads)
{
	int64_t b = (n + threads - 1) / threads;
	return (int)(b < 1 ? 1 : b);
}

// Launch accounting: every kernel launch of the library goes through
// M3G_LAUNCH, which counts it and, when the kernel's name is the one selected
// with m3d_gpu_profiler_reset, brackets it with CUDA events on its stream.
void launchBegin(const char* name, cudaStream_t s);
void launchEnd(const char* name, cudaStream_t s);

// Counts one device allocation (every cudaMalloc of the library calls it);
// read by m3d_gpu_profiler_allocations.
void countAllocation();

// Every async copy of the library goes through this wrapper (see the macro
// below), which adds host->device and device->host bytes to the counters
// read by m3d_gpu_profiler_bytes.
cudaError_t countedMemcpyAsync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s);

} // namespace m3g

#define cudaMemcpyAsync(...) ::m3g::countedMemcpyAsync(__VA_ARGS__)

namespace m3g
{

// Programmatic dependent launch.  Every kernel of the library is launched
// with programmatic stream serialisation allowed, so the next kernel of the
// stream is scheduled while this one's last blocks still run and its launch
// latency hides behind them.  Every kernel therefore begins with
// M3G_KERNEL_BEGIN: griddepcontrol.wait holds it until the previous grid of
// the stream has completed and its writes are visible (a no-op when the
// launch had no programmatic dependency), then launch_dependents lets the
// next grid be scheduled.  Because every grid waits before touching memory,
// each one also starts after every earlier grid of the stream has completed,
// as without the attribute.
__device__ __forceinline__ void gridDependencyWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void gridLaunchDependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... Params, typename... Args>
inline void launchProgrammatic(void (*kern)(Params...), dim3 grid, dim3 block, cudaStream_t stream, Args&&... args)
{
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = 1;
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = 0;
	cfg.stream = stream;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	cudaLaunchKernelEx(&cfg, kern, static_cast<Args&&>(args)...);
}

} // namespace m3g

#define M3G_KERNEL_BEGIN()                                                                                             \
	do                                                                                                                 \
	{                                                                                                                  \
		::m3g::gridDependencyWait();                                                                                   \
		::m3g::gridLaunchDependents();                                                                                 \
	} while (0)

// the same, accounted under an explicit name (template instances of one kernel)
#define M3G_LAUNCH_AS(name, kern, grid, block, stream, ...)                                                            \
	do                                                                                                                 \
	{                                                                                                                  \
		::m3g::launchBegin(name, (stream));                                                                           \
		::m3g::launchProgrammatic(kern, dim3(grid), dim3(block), (stream), __VA_ARGS__);                              \
		::m3g::launchEnd(name, (stream));                                                                             \
	} while (0)

#define M3G_LAUNCH(kern, grid, block, stream, ...)                                                                     \
	do                                                                                                                 \
	{                                                                                                                  \
		::m3g::launchBegin(#kern, (stream));                                                                          \
		::m3g::launchProgrammatic(kern, dim3(grid), dim3(block), (stream), __VA_ARGS__);                              \
		::m3g::launchEnd(#kern, (stream));                                                                            \
	} while (0)

// Broadphase and contact bookkeeping of one step:
//   fat-AABB refresh -> active/stable cell entries -> stable radix sort ->
//   cell runs -> pair enumeration with the admission filters -> oversized
//   pairs -> first-occurrence dedupe -> contact creation -> removal of pairs
//   whose fat boxes separated.
//
// Contact ORDER is part of the result (the Gauss-Seidel solver and the graph
// colouring follow it), so every stage reproduces the reference's order:
// pairs are emitted cell run by cell run (runs in ascending cell key), inside
// a run active x active pairs in (i, j > i) entry order and then active x
// stable pairs stable-entry-major, then the oversized loops; a pair already
// present (before the step or earlier in the stream) is skipped; removal is
// the closed form of the reference's descending swap-remove.
// (reference src/world.cpp:156-229, 1456-1735; src/grid.cpp:19-95)
#include "m3d_collide.cuh"
#include "m3d_dev.cuh"

namespace m3g
{

__device__ __forceinline__ int64_t cellCoord(float v, float inv) { return (int64_t)floorf(v * inv); }

// PackCell (reference src/grid.cpp:19-37): each coordinate offset by half its
// range and masked to `bits` bits, x above y above z, so keys order cells as
// (x, y, z).  One world uses 21 bits per coordinate, as the reference; a
// batch of worlds puts the world index above the coordinates (fewer bits
// each), which orders entries world-major and, inside a world, exactly as the
// world's own keys do while its cells stay within the narrower range.
__device__ __forceinline__ uint64_t packCell(int64_t x, int64_t y, int64_t z, uint32_t world, int bits)
{
	const int64_t offset = (int64_t)1 << (bits - 1);
	const uint64_t mask = (1ull << bits) - 1ull;
	uint64_t ux = (uint64_t)(x + offset) & mask;
	uint64_t uy = (uint64_t)(y + offset) & mask;
	uint64_t uz = (uint64_t)(z + offset) & mask;
	return ((uint64_t)world << (3 * bits)) | (ux << (2 * bits)) | (uy << bits) | uz;
}

__device__ __forceinline__ uint64_t cellKeyOf(V3 p, float inv, uint32_t world, int bits)
{
	return packCell(cellCoord(p.x, inv), cellCoord(p.y, inv), cellCoord(p.z, inv), world, bits);
}

__device__ __forceinline__ uint64_t pairKey(int32_t lo, int32_t hi)
{
	return ((uint64_t)(uint32_t)lo << 32) | (uint64_t)(uint32_t)hi;
}

__device__ __forceinline__ Box loadFat(const BodySoA& B, int i)
{
	Box b;
	b.lo = ld3(B.fatLo[i]);
	b.hi = ld3(B.fatHi[i]);
	return b;
}

// cells covered by a fat box; > kOversizedCellSpan means "coarse list"
__device__ __forceinline__ int64_t cellSpan(const Box& b, float inv)
{
	int64_t x0 = cellCoord(b.lo.x, inv), y0 = cellCoord(b.lo.y, inv), z0 = cellCoord(b.lo.z, inv);
	int64_t x1 = cellCoord(b.hi.x, inv), y1 = cellCoord(b.hi.y, inv), z1 = cellCoord(b.hi.z, inv);
	return (x1 - x0 + 1) * (y1 - y0 + 1) * (z1 - z0 + 1);
}

// ---------------------------------------------------------------------------
// fat AABB refresh (reference src/world.cpp:143-211)
// ---------------------------------------------------------------------------

// rebuildAny: the stable tier is emitted this step; worldRebuild (batch only)
// says which worlds rebuild theirs, the others keep their entries.
__global__ void kRefresh(BodySoA B, int32_t n, float dt, int rebuildAny, const uint8_t* worldRebuild, float inv,
						 uint32_t* cntA, uint32_t* overA, uint32_t* cntS, uint32_t* overS, uint8_t* inActiveCells)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	const bool rebuildStable = rebuildAny && (worldRebuild == nullptr || worldRebuild[worldOfBody(B, i)] != 0);
	uint8_t st = B.state[i];
	bool inUse = (st & kStInUse) != 0;
	bool awake = (st & kStAwake) != 0;
	const BodyCold& cold = B.cold[i];
	bool stable = inUse && !awake;
	bool active = inUse && (awake || !B.inStableTier[i]);
	B.isActive[i] = active ? 1 : 0;
	B.isStable[i] = stable ? 1 : 0;
	B.moved[i] = 0;
	B.bFlags[i] = (uint8_t)((inUse ? kBFInUse : 0) | ((inUse && cold.type == kDynamic) ? kBFDynamic : 0) |
							((inUse && cold.type == kKinematic) ? kBFKinematic : 0) | (awake ? kBFAwake : 0));
	V3 margin = v3(kAABBMargin, kAABBMargin, kAABBMargin);
	if (active)
	{
		Box pred = shapeAABB(cold.shape, bodyXf(B, i));
		V3 vel = ld3(B.vel[i]);
		V3 stp = scale(dt, vel);
		if (stp.x < 0.0f) pred.lo.x += stp.x; else pred.hi.x += stp.x;
		if (stp.y < 0.0f) pred.lo.y += stp.y; else pred.hi.y += stp.y;
		if (stp.z < 0.0f) pred.lo.z += stp.z; else pred.hi.z += stp.z;
		if (!B.hasFat[i] || !contains(loadFat(B, i), pred))
		{
			Box fat;
			fat.lo = sub(pred.lo, margin);
			fat.hi = add(pred.hi, margin);
			V3 slack = scale(2.0f * dt, vel);
			if (slack.x < 0.0f) fat.lo.x += slack.x; else fat.hi.x += slack.x;
			if (slack.y < 0.0f) fat.lo.y += slack.y; else fat.hi.y += slack.y;
			if (slack.z < 0.0f) fat.lo.z += slack.z; else fat.hi.z += slack.z;
			B.fatLo[i] = st3(fat.lo);
			B.fatHi[i] = st3(fat.hi);
			B.hasFat[i] = 1;
			B.moved[i] = 1;
		}
	}
	else if (stable && rebuildStable && !B.hasFat[i])
	{
		Box box = shapeAABB(cold.shape, bodyXf(B, i));
		box.lo = sub(box.lo, margin);
		box.hi = add(box.hi, margin);
		V3 d = scale(dt, ld3(B.vel[i]));
		if (d.x < 0.0f) box.lo.x += d.x; else box.hi.x += d.x;
		if (d.y < 0.0f) box.lo.y += d.y; else box.hi.y += d.y;
		if (d.z < 0.0f) box.lo.z += d.z; else box.hi.z += d.z;
		B.fatLo[i] = st3(box.lo);
		B.fatHi[i] = st3(box.hi);
		B.hasFat[i] = 1;
	}

	// tier membership and cell counts (reference src/grid.cpp:39-78)
	uint32_t ca = 0, oa = 0;
	uint8_t inCellsA = 0;
	if (active)
	{
		int64_t span = cellSpan(loadFat(B, i), inv);
		if (span > kOversizedCellSpan)
		{
			oa = 1;
		}
		else
		{
			ca = (uint32_t)span;
			inCellsA = 1;
		}
	}
	cntA[i] = ca;
	overA[i] = oa;
	inActiveCells[i] = inCellsA;
	if (rebuildAny && !rebuildStable)
	{
		cntS[i] = 0; // this body's world keeps its stable entries
		overS[i] = 0;
	}
	if (rebuildStable)
	{
		uint32_t cs = 0, os = 0;
		uint8_t inCellsS = 0;
		if (stable)
		{
			int64_t span = cellSpan(loadFat(B, i), inv);
			if (span > kOversizedCellSpan)
			{
				os = 1;
			}
			else
			{
				cs = (uint32_t)span;
				inCellsS = 1;
			}
		}
		cntS[i] = cs;
		overS[i] = os;
		B.inStableCells[i] = inCellsS;
		B.inStableTier[i] = stable ? 1 : 0;
	}
}

void launchRefresh(DevWorld& w, int32_t n, float dt, bool rebuildStable, float cellSize)
{
	float inv = 1.0f / cellSize;
	size_t n4 = (size_t)(n + 1) * sizeof(uint32_t);
	w.cellCountA.ensure(n4);
	w.overFlagA.ensure(n4);
	w.cellCountS.ensure(n4);
	w.overFlagS.ensure(n4);
	w.inActiveCells.ensure((size_t)n + 1);
	if (n <= 0)
	{
		return;
	}
	M3G_LAUNCH(kRefresh, blocksFor(n, 256), 256, w.stream, w.B, n, dt, rebuildStable ? 1 : 0,
			   w.batched ? w.worldRebuild.as<uint8_t>() : nullptr, inv,
													   w.cellCountA.as<uint32_t>(), w.overFlagA.as<uint32_t>(),
													   w.cellCountS.as<uint32_t>(), w.overFlagS.as<uint32_t>(),
													   w.inActiveCells.as<uint8_t>());
}

// ---------------------------------------------------------------------------
// tier build: entries (cell key, body) in body order, then a stable sort by
// key, which yields the unique (key, body) order (reference src/grid.cpp:39-95)
// ---------------------------------------------------------------------------

__global__ void kEmitEntries(BodySoA B, int32_t n, float inv, int bits, const uint32_t* cnt, const uint32_t* offs,
							 uint64_t* keys, uint32_t* vals, uint32_t* ranges)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	uint32_t lo[4] = { 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu }, hi[4] = { 0u, 0u, 0u, 0u };
	const uint64_t mask = (1ull << bits) - 1ull;
	if (i < n && cnt[i] != 0)
	{
		Box b = loadFat(B, i);
		int64_t x0 = cellCoord(b.lo.x, inv), y0 = cellCoord(b.lo.y, inv), z0 = cellCoord(b.lo.z, inv);
		int64_t x1 = cellCoord(b.hi.x, inv), y1 = cellCoord(b.hi.y, inv), z1 = cellCoord(b.hi.z, inv);
		uint32_t o = offs[i];
		const uint32_t world = worldOfBody(B, i);
		for (int64_t x = x0; x <= x1; ++x)
		{
			for (int64_t y = y0; y <= y1; ++y)
			{
				for (int64_t z = z0; z <= z1; ++z)
				{
					uint64_t k = packCell(x, y, z, world, bits);
					keys[o] = k;
					vals[o] = (uint32_t)i;
					uint32_t f[4] = { world, (uint32_t)((k >> (2 * bits)) & mask), (uint32_t)((k >> bits) & mask),
									  (uint32_t)(k & mask) };
#pragma unroll
					for (int a = 0; a < 4; ++a)
					{
						lo[a] = f[a] < lo[a] ? f[a] : lo[a];
						hi[a] = f[a] > hi[a] ? f[a] : hi[a];
					}
					++o;
				}
			}
		}
	}
	// the range of each key field decides which radix passes run
#pragma unroll
	for (int a = 0; a < 4; ++a)
	{
		uint32_t l = lo[a], h = hi[a];
		for (int off = 16; off > 0; off >>= 1)
		{
			uint32_t lt = __shfl_xor_sync(0xffffffffu, l, off);
			uint32_t ht = __shfl_xor_sync(0xffffffffu, h, off);
			l = lt < l ? lt : l;
			h = ht > h ? ht : h;
		}
		if ((threadIdx.x & 31) == 0 && l <= h)
		{
			atomicMin(&ranges[a], l);
			atomicMax(&ranges[4 + a], h);
		}
	}
}

__global__ void kCompactIndices(const uint32_t* flags, const uint32_t* offs, int32_t n, int32_t* out)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && flags[i])
	{
		out[offs[i]] = i;
	}
}

// per tier: min of (world, x, y, z) fields, then their max
__global__ void kInitRanges(uint32_t* ranges)
{
	M3G_KERNEL_BEGIN();
	for (int t = 0; t < 2; ++t)
	{
		for (int a = 0; a < 4; ++a)
		{
			ranges[8 * t + a] = 0xFFFFFFFFu;
			ranges[8 * t + 4 + a] = 0u;
		}
	}
}

// Radix-sort parameters of one tier from its key-field ranges: subtracting
// each field's minimum keeps the key order (no field borrows from the next)
// and leaves only the low bits of each field varying.
static void tierSortBias(const uint32_t* r, int keyBits, uint64_t* bias, uint64_t* vary)
{
	uint64_t b = 0ull, v = 0ull;
	for (int a = 0; a < 4; ++a)
	{
		const int shift = keyBits * (3 - a);
		if (r[a] > r[4 + a])
		{
			continue; // no entries
		}
		uint32_t d = r[4 + a] - r[a];
		int bits = 0;
		while (bits < 32 && (d >> bits) != 0)
		{
			++bits;
		}
		b |= (uint64_t)r[a] << shift;
		v |= (bits >= 64 ? ~0ull : ((1ull << bits) - 1ull)) << shift;
	}
	*bias = b;
	*vary = v;
}

// One tier: counts -> offsets -> (key, body) entries in body order and the
// oversized list.  Entry buffers are sized by the bound of 64 cells per body,
// so nothing waits for the host; the sort runs after the step's first sync.
static void emitTier(DevWorld& w, int32_t n, float inv, DevBuf& cnt, DevBuf& over, DevBuf& offs, DevBuf& ooffs,
					 DevBuf& keys, DevBuf& vals, DevBuf& overList, uint32_t* entryTotal, uint32_t* overTotal,
					 uint32_t* ranges, size_t extra = 0)
{
	size_t bound = (size_t)n * kOversizedCellSpan + 1 + extra;
	offs.ensure((size_t)(n + 1) * sizeof(uint32_t));
	ooffs.ensure((size_t)(n + 1) * sizeof(uint32_t));
	keys.ensure(bound * sizeof(uint64_t));
	vals.ensure(bound * sizeof(uint32_t));
	overList.ensure((size_t)(n + 1) * sizeof(int32_t));
	scanExclusive2(cnt.as<uint32_t>(), offs.as<uint32_t>(), n, entryTotal, over.as<uint32_t>(), ooffs.as<uint32_t>(), n,
				   overTotal, w.prim, w.stream);
	if (n > 0)
	{
		M3G_LAUNCH(kEmitEntries, blocksFor(n, 128), 128, w.stream, w.B, n, inv, w.keyBits, cnt.as<uint32_t>(),
				   offs.as<uint32_t>(), keys.as<uint64_t>(), vals.as<uint32_t>(), ranges);
		M3G_LAUNCH(kCompactIndices, blocksFor(n, 256), 256, w.stream, over.as<uint32_t>(), ooffs.as<uint32_t>(), n,
				   overList.as<int32_t>());
	}
}

void launchEmitGrid(DevWorld& w, int32_t n, float cellSize, bool rebuildStable)
{
	StepCounters* dc = devCounters(w);
	w.keyRanges.ensure(16 * sizeof(uint32_t));
	uint32_t* ranges = w.keyRanges.as<uint32_t>();
	M3G_LAUNCH(kInitRanges, 1, 1, w.stream, ranges);
	float inv = 1.0f / cellSize;
	emitTier(w, n, inv, w.cellCountA, w.overFlagA, w.entryOffsA, w.overOffsA, w.activeKeys, w.activeVals, w.activeOver,
			 &dc->activeEntries, &dc->activeOversized, ranges);
	if (rebuildStable)
	{
		size_t extra = 0;
		if (w.batched)
		{
			// worlds that keep their stable tier: entries set aside before the
			// fresh ones overwrite the arrays, appended back after the sync
			launchKeepStable(w, ranges + 8);
			extra = (size_t)w.stableEntries;
		}
		emitTier(w, n, inv, w.cellCountS, w.overFlagS, w.entryOffsS, w.overOffsS, w.stableKeys, w.stableVals,
				 w.stableOver, &dc->stableEntries, &dc->stableOversized, ranges + 8, extra);
	}
	if (w.hostRanges == nullptr)
	{
		cudaMallocHost((void**)&w.hostRanges, 16 * sizeof(uint32_t));
	}
	cudaMemcpyAsync(w.hostRanges, ranges, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, w.stream);
}

// after the first sync of the step: sizes and key ranges are on the host
void launchSortGrid(DevWorld& w, bool rebuildStable)
{
	const StepCounters* hc = w.hostCounters;
	uint64_t bias, vary;
	w.activeEntries = hc->activeEntries;
	w.activeOverCount = (int32_t)hc->activeOversized;
	if (w.activeEntries > 1)
	{
		tierSortBias(w.hostRanges, w.keyBits, &bias, &vary);
		radixSortPairs(w.activeKeys.as<uint64_t>(), w.activeVals.as<uint32_t>(), w.activeEntries, vary, w.prim,
					   w.stream, nullptr, bias);
	}
	if (rebuildStable)
	{
		w.stableEntries = hc->stableEntries;
		w.stableOverCount = (int32_t)hc->stableOversized;
		if (w.batched)
		{
			launchAppendKeptStable(w, hc->stableEntries, (int32_t)hc->stableOversized);
		}
		if (w.stableEntries > 1)
		{
			tierSortBias(w.hostRanges + 8, w.keyBits, &bias, &vary);
			radixSortPairs(w.stableKeys.as<uint64_t>(), w.stableVals.as<uint32_t>(), w.stableEntries, vary, w.prim,
						   w.stream, nullptr, bias);
		}
	}
}

// ---------------------------------------------------------------------------
// cell runs over the sorted active entries (reference src/world.cpp:1576-1587)
// ---------------------------------------------------------------------------

__global__ void kRunFlags(const uint64_t* keys, int64_t n, uint32_t* flag)
{
	M3G_KERNEL_BEGIN();
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
	}
}

__global__ void kRunStarts(const uint32_t* flag, const uint32_t* offs, int64_t n, int32_t* starts, const uint32_t* total)
{
	M3G_KERNEL_BEGIN();
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && flag[i])
	{
		starts[offs[i]] = (int32_t)i;
	}
	if (i == 0)
	{
		starts[*total] = (int32_t)n;
	}
}

void launchFindRuns(DevWorld& w)
{
	StepCounters* dc = devCounters(w);
	int64_t n = w.activeEntries;
	w.runFlag.ensure((size_t)(n + 1) * sizeof(uint32_t));
	w.runOffs.ensure((size_t)(n + 1) * sizeof(uint32_t));
	w.runStarts.ensure((size_t)(n + 2) * sizeof(int32_t));
	w.runCount = (int32_t)n; // upper bound; the exact count stays on the device
	if (n <= 0)
	{
		fillWords(&dc->runs, 0u, sizeof(uint32_t), w.stream);
		return;
	}
	M3G_LAUNCH(kRunFlags, blocksFor(n, 256), 256, w.stream, w.activeKeys.as<uint64_t>(), n, w.runFlag.as<uint32_t>());
	uint32_t* offs = w.runOffs.as<uint32_t>();
	scanExclusive(w.runFlag.as<uint32_t>(), offs, n, &dc->runs, w.prim, w.stream);
	M3G_LAUNCH(kRunStarts, blocksFor(n, 256), 256, w.stream, w.runFlag.as<uint32_t>(), offs, n, w.runStarts.as<int32_t>(),
			   &dc->runs);
}

// ---------------------------------------------------------------------------
// pair enumeration (reference src/world.cpp:1486-1641, 1663-1702)
// ---------------------------------------------------------------------------

struct PairCtx
{
	BodySoA B;
	const uint64_t* existing;
	uint32_t existingMask;
	const uint64_t* jointed;
	int32_t jointedCount;
	float inv;
	int keyBits;
};

__device__ __forceinline__ bool jointedContains(const uint64_t* keys, int32_t n, uint64_t k)
{
	int32_t lo = 0, hi = n;
	while (lo < hi)
	{
		int32_t mid = (lo + hi) >> 1;
		if (keys[mid] < k)
		{
			lo = mid + 1;
		}
		else
		{
			hi = mid;
		}
	}
	return lo < n && keys[lo] == k;
}

// every read-only admission filter of the reference (src/world.cpp:1486-1538)
__device__ bool admissible(const PairCtx& P, int32_t a, int32_t b, uint64_t* keyOut)
{
	if (a == b || worldOfBody(P.B, a) != worldOfBody(P.B, b))
	{
		return false;
	}
	if (!P.B.moved[a] && !P.B.moved[b])
	{
		return false;
	}
	int32_t lo = a < b ? a : b;
	int32_t hi = a < b ? b : a;
	uint8_t sl = P.B.state[lo], sh = P.B.state[hi];
	if (!(sl & kStInUse) || !(sh & kStInUse))
	{
		return false;
	}
	const BodyCold& cl = P.B.cold[lo];
	const BodyCold& ch = P.B.cold[hi];
	if (cl.type != kDynamic && ch.type != kDynamic)
	{
		return false;
	}
	if (!(sl & kStAwake) && !(sh & kStAwake))
	{
		return false;
	}
	if (!overlap(loadFat(P.B, lo), loadFat(P.B, hi)))
	{
		return false;
	}
	if (cl.groupIndex != 0 && cl.groupIndex == ch.groupIndex)
	{
		if (cl.groupIndex < 0)
		{
			return false;
		}
	}
	else if ((cl.categoryBits & ch.maskBits) == 0 || (ch.categoryBits & cl.maskBits) == 0)
	{
		return false;
	}
	uint64_t key = pairKey(lo, hi);
	if (hashContains(P.existing, P.existingMask, key))
	{
		return false;
	}
	if (P.jointedCount > 0 && jointedContains(P.jointed, P.jointedCount, key))
	{
		return false;
	}
	*keyOut = key;
	return true;
}

__device__ __forceinline__ int64_t lowerBoundKey(const uint64_t* keys, int64_t n, uint64_t k)
{
	int64_t lo = 0, hi = n;
	while (lo < hi)
	{
		int64_t mid = (lo + hi) >> 1;
		if (keys[mid] < k)
		{
			lo = mid + 1;
		}
		else
		{
			hi = mid;
		}
	}
	return lo;
}

// One thread per cell run: count (EMIT=false) or write (EMIT=true) the
// admitted pair keys of the run in the reference's enumeration order.
template <bool EMIT>
__global__ void kRunPairs(PairCtx P, const uint64_t* actKeys, const uint32_t* actVals, const int32_t* runStarts,
						  int32_t runMax, const uint32_t* runsDev, const uint64_t* stabKeys, const uint32_t* stabVals,
						  int64_t stabCount, uint32_t* counts, const uint32_t* offsets, uint64_t* out)
{
	M3G_KERNEL_BEGIN();
	int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= runMax)
	{
		return;
	}
	if (r >= (int)*runsDev)
	{
		if (!EMIT)
		{
			counts[r] = 0; // past the last run: contributes nothing to the scan
		}
		return;
	}
	int32_t s = runStarts[r], e = runStarts[r + 1];
	uint64_t key = actKeys[s];
	uint32_t k = EMIT ? offsets[r] : 0u;
	for (int32_t i = s; i < e; ++i)
	{
		int32_t a = (int32_t)actVals[i];
		V3 la = ld3(P.B.fatLo[a]);
		for (int32_t j = i + 1; j < e; ++j)
		{
			int32_t b = (int32_t)actVals[j];
			V3 lo2 = vmax(la, ld3(P.B.fatLo[b]));
			uint64_t pk;
			if (cellKeyOf(lo2, P.inv, worldOfBody(P.B, a), P.keyBits) == key && admissible(P, a, b, &pk))
			{
				if (EMIT)
				{
					out[k] = pk;
				}
				++k;
			}
		}
	}
	for (int64_t t = lowerBoundKey(stabKeys, stabCount, key); t < stabCount && stabKeys[t] == key; ++t)
	{
		int32_t b = (int32_t)stabVals[t];
		V3 lb = ld3(P.B.fatLo[b]);
		for (int32_t i = s; i < e; ++i)
		{
			int32_t a = (int32_t)actVals[i];
			if (a == b)
			{
				continue; // stale stable entry of a body that woke
			}
			V3 lo2 = vmax(ld3(P.B.fatLo[a]), lb);
			uint64_t pk;
			if (cellKeyOf(lo2, P.inv, worldOfBody(P.B, a), P.keyBits) == key && admissible(P, a, b, &pk))
			{
				if (EMIT)
				{
					out[k] = pk;
				}
				++k;
			}
		}
	}
	if (!EMIT)
	{
		counts[r] = k;
	}
}

// Oversized pairs, flattened in the reference's loop order:
//   for each active oversized a (list order): every in-grid body b != a, then
//   the later active oversized bodies, then every stable oversized b != a;
//   then for each stable oversized a: every body in active cells.
struct OverCtx
{
	const int32_t* actOver;
	int32_t nAO;
	const int32_t* stabOver;
	int32_t nSO;
	int32_t n;
	const uint8_t* inActiveCells;
};

__device__ bool overCandidate(const OverCtx& O, int64_t idx, int32_t* aOut, int32_t* bOut)
{
	for (int32_t oi = 0; oi < O.nAO; ++oi)
	{
		int32_t a = O.actOver[oi];
		int64_t blk = (int64_t)O.n + (O.nAO - oi - 1) + O.nSO;
		if (idx < blk)
		{
			int32_t b;
			if (idx < O.n)
			{
				b = (int32_t)idx;
				if (b == a)
				{
					return false;
				}
				*aOut = a;
				*bOut = b;
				return true; // in-grid test done by the caller
			}
			idx -= O.n;
			if (idx < O.nAO - oi - 1)
			{
				*aOut = a;
				*bOut = O.actOver[oi + 1 + idx];
				return true;
			}
			idx -= O.nAO - oi - 1;
			b = O.stabOver[idx];
			if (b == a)
			{
				return false;
			}
			*aOut = a;
			*bOut = b;
			return true;
		}
		idx -= blk;
	}
	int64_t si = idx / O.n;
	int32_t b = (int32_t)(idx - si * O.n);
	if (!O.inActiveCells[b])
	{
		return false;
	}
	*aOut = O.stabOver[si];
	*bOut = b;
	return true;
}

__global__ void kOverPairs(PairCtx P, OverCtx O, int64_t total, uint32_t* flags, uint64_t* keys)
{
	M3G_KERNEL_BEGIN();
	int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= total)
	{
		return;
	}
	int32_t a, b;
	uint32_t ok = 0;
	uint64_t pk = 0;
	if (overCandidate(O, idx, &a, &b))
	{
		// first segment of an active oversized body: only bodies in either grid
		bool gridOnly = false;
		{
			int64_t j = idx;
			for (int32_t oi = 0; oi < O.nAO; ++oi)
			{
				int64_t blk = (int64_t)O.n + (O.nAO - oi - 1) + O.nSO;
				if (j < blk)
				{
					gridOnly = j < O.n;
					break;
				}
				j -= blk;
			}
		}
		bool inGrid = !gridOnly || O.inActiveCells[b] || P.B.inStableCells[b];
		if (inGrid && admissible(P, a, b, &pk))
		{
			ok = 1;
		}
	}
	flags[idx] = ok;
	keys[idx] = pk;
}

__global__ void kScatterKeys(const uint32_t* flags, const uint32_t* offs, const uint64_t* keys, int64_t n, uint64_t* out)
{
	M3G_KERNEL_BEGIN();
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && flags[i])
	{
		out[offs[i]] = keys[i];
	}
}

__global__ void kInsertExisting(const int2* bodies, int32_t count, uint64_t* table, uint32_t mask, uint32_t* fail)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= count)
	{
		return;
	}
	int2 ab = bodies[c];
	if (hashInsert(table, mask, pairKey(ab.x, ab.y)) == 0xFFFFFFFFu)
	{
		atomicAdd(fail, 1u);
	}
}

// first occurrence of each key in the admitted stream wins
__global__ void kDedupeMark(const uint64_t* keys, int64_t n, uint64_t* table, uint32_t* pos, uint32_t mask,
							uint32_t* fail)
{
	M3G_KERNEL_BEGIN();
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	uint32_t slot = hashInsert(table, mask, keys[i]);
	if (slot == 0xFFFFFFFFu)
	{
		atomicAdd(fail, 1u);
		return;
	}
	atomicMin(&pos[slot], (uint32_t)i);
}

__device__ __forceinline__ uint32_t hashFind(const uint64_t* table, uint32_t capMask, uint64_t key)
{
	uint32_t slot = hashKey(key) & capMask;
	for (uint32_t probe = 0; probe <= capMask; ++probe)
	{
		uint64_t k = table[slot];
		if (k == key)
		{
			return slot;
		}
		if (k == kEmptyKey)
		{
			return 0xFFFFFFFFu;
		}
		slot = (slot + 1) & capMask;
	}
	return 0xFFFFFFFFu;
}

__global__ void kDedupeKeep(const uint64_t* keys, int64_t n, const uint64_t* table, const uint32_t* pos, uint32_t mask,
							uint32_t* keep)
{
	M3G_KERNEL_BEGIN();
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	uint32_t slot = hashFind(table, mask, keys[i]);
	keep[i] = (slot != 0xFFFFFFFFu && pos[slot] == (uint32_t)i) ? 1u : 0u;
}

static uint32_t tableCapacity(int64_t keys)
{
	uint64_t cap = 1024;
	while (cap < (uint64_t)keys * 2 + 16)
	{
		cap <<= 1;
	}
	return (uint32_t)cap;
}

static PairCtx pairCtx(DevWorld& w, float cellSize)
{
	PairCtx P;
	P.B = w.B;
	P.existing = w.existingSet.as<uint64_t>();
	P.existingMask = w.existingMask;
	P.jointed = w.jointedPairs.as<uint64_t>();
	P.jointedCount = w.jointedCount;
	P.inv = 1.0f / cellSize;
	P.keyBits = w.keyBits;
	return P;
}

static OverCtx overCtx(DevWorld& w, int32_t n, int64_t* total)
{
	OverCtx O;
	O.actOver = w.activeOver.as<int32_t>();
	O.nAO = w.activeOverCount;
	O.stabOver = w.stableOver.as<int32_t>();
	O.nSO = w.stableOverCount;
	O.n = n;
	O.inActiveCells = w.inActiveCells.as<uint8_t>();
	*total = (int64_t)O.nAO * ((int64_t)n + O.nSO) + (int64_t)O.nAO * (O.nAO - 1) / 2 + (int64_t)O.nSO * n;
	return O;
}

// ---- oversized pairs, world by world ---------------------------------------------
// The reference's oversized loops (src/world.cpp:1663-1702) pair an oversized
// body with every body of its world.  In a batch the candidate stream is cut
// into one block per oversized body - in the order of the single-world loops
// (active oversized bodies, then stable ones) - holding only its own world's
// bodies, so the stream of each world is the one its own step produces.

__device__ __forceinline__ int32_t lowerBoundI32(const int32_t* a, int32_t n, int32_t v)
{
	int32_t lo = 0, hi = n;
	while (lo < hi)
	{
		int32_t mid = (lo + hi) >> 1;
		if (a[mid] < v)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo;
}

struct OverBatch
{
	const int32_t* actOver;
	int32_t nAO;
	const int32_t* stabOver;
	int32_t nSO;
	const uint32_t* first; // per world + 1: first body slot
	const uint8_t* inActiveCells;
	const uint32_t* blockOffs;
};

__global__ void kOverBlocks(const BodySoA B, OverBatch O, uint32_t* blocks)
{
	M3G_KERNEL_BEGIN();
	int o = blockIdx.x * blockDim.x + threadIdx.x;
	if (o >= O.nAO + O.nSO)
	{
		return;
	}
	const int32_t a = o < O.nAO ? O.actOver[o] : O.stabOver[o - O.nAO];
	const uint32_t w = worldOfBody(B, a);
	const int32_t f0 = (int32_t)O.first[w], f1 = (int32_t)O.first[w + 1];
	uint32_t size = (uint32_t)(f1 - f0);
	if (o < O.nAO)
	{
		const int32_t aEnd = lowerBoundI32(O.actOver, O.nAO, f1);
		const int32_t s0 = lowerBoundI32(O.stabOver, O.nSO, f0), s1 = lowerBoundI32(O.stabOver, O.nSO, f1);
		size += (uint32_t)(aEnd - o - 1) + (uint32_t)(s1 - s0);
	}
	blocks[o] = size;
}

__global__ void kOverPairsBatch(PairCtx P, OverBatch O, int64_t maxTotal, const uint32_t* totalDev, uint32_t* flags,
								uint64_t* keys)
{
	M3G_KERNEL_BEGIN();
	const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= maxTotal)
	{
		return;
	}
	uint32_t ok = 0;
	uint64_t pk = 0;
	if (idx < (int64_t)*totalDev)
	{
		// the block holding idx: the last o with blockOffs[o] <= idx
		int32_t lo = 0, hi = O.nAO + O.nSO;
		while (hi - lo > 1)
		{
			int32_t mid = (lo + hi) >> 1;
			if ((int64_t)O.blockOffs[mid] <= idx)
				lo = mid;
			else
				hi = mid;
		}
		const int32_t o = lo;
		int64_t local = idx - (int64_t)O.blockOffs[o];
		const int32_t a = o < O.nAO ? O.actOver[o] : O.stabOver[o - O.nAO];
		const uint32_t w = worldOfBody(P.B, a);
		const int32_t f0 = (int32_t)O.first[w], f1 = (int32_t)O.first[w + 1];
		const int64_t nw = f1 - f0;
		int32_t b = -1;
		bool inGrid = true;
		if (o < O.nAO)
		{
			if (local < nw)
			{
				b = f0 + (int32_t)local;
				inGrid = O.inActiveCells[b] || P.B.inStableCells[b];
			}
			else
			{
				local -= nw;
				const int32_t aEnd = lowerBoundI32(O.actOver, O.nAO, f1);
				if (local < aEnd - o - 1)
				{
					b = O.actOver[o + 1 + local];
				}
				else
				{
					local -= aEnd - o - 1;
					b = O.stabOver[lowerBoundI32(O.stabOver, O.nSO, f0) + local];
				}
			}
		}
		else
		{
			b = f0 + (int32_t)local;
			inGrid = O.inActiveCells[b] != 0;
		}
		if (b >= 0 && b != a && inGrid && admissible(P, a, b, &pk))
		{
			ok = 1;
		}
	}
	flags[idx] = ok;
	keys[idx] = pk;
}

int64_t launchOverPairsBatch(DevWorld& w, const PairCtx& P)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	const int32_t nAO = w.activeOverCount, nSO = w.stableOverCount, nO = nAO + nSO;
	if (nO == 0)
	{
		setDeviceCount(w, &dc->overPairs, 0u);
		return 0;
	}
	const int64_t maxN = w.maxWorldBodies;
	const int64_t maxTotal = (int64_t)nO * (maxN + (nO < maxN ? nO : maxN));
	w.overBlockOffs.ensure((size_t)(nO + 2) * sizeof(uint32_t));
	w.overBlockCount.ensure((size_t)(nO + 2) * sizeof(uint32_t));
	w.overFlag.ensure((size_t)(maxTotal + 1) * sizeof(uint32_t));
	w.overScan.ensure((size_t)(maxTotal + 1) * sizeof(uint32_t));
	w.overKeys.ensure((size_t)(maxTotal + 1) * sizeof(uint64_t));
	OverBatch O;
	O.actOver = w.activeOver.as<int32_t>();
	O.nAO = nAO;
	O.stabOver = w.stableOver.as<int32_t>();
	O.nSO = nSO;
	O.first = w.worldFirstBody.as<uint32_t>();
	O.inActiveCells = w.inActiveCells.as<uint8_t>();
	O.blockOffs = w.overBlockOffs.as<uint32_t>();
	uint32_t* blocks = w.overBlockCount.as<uint32_t>();
	M3G_LAUNCH(kOverBlocks, blocksFor(nO, 256), 256, s, w.B, O, blocks);
	uint32_t* total = w.overBlockOffs.as<uint32_t>() + nO;
	scanExclusive(blocks, w.overBlockOffs.as<uint32_t>(), nO, total, w.prim, s);
	M3G_LAUNCH(kOverPairsBatch, blocksFor(maxTotal, 256), 256, s, P, O, maxTotal, total, w.overFlag.as<uint32_t>(),
			   w.overKeys.as<uint64_t>());
	scanExclusive(w.overFlag.as<uint32_t>(), w.overScan.as<uint32_t>(), maxTotal, &dc->overPairs, w.prim, s);
	return maxTotal;
}

// Count the admitted pairs of every cell run and of the oversized loops; the
// step's second sync reads the two totals.
void launchPairCount(DevWorld& w, int32_t n, float cellSize)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;

	// existing contact keys
	uint32_t ecap = tableCapacity(w.contactCount);
	w.existingSet.ensure((size_t)ecap * sizeof(uint64_t));
	w.existingMask = ecap - 1;
	fillWords(w.existingSet.ptr, 0xFFFFFFFFu, (size_t)ecap * sizeof(uint64_t), s);
	if (w.contactCount > 0)
	{
		M3G_LAUNCH(kInsertExisting, blocksFor(w.contactCount, 256), 256, s, w.C.bodies, w.contactCount,
				   w.existingSet.as<uint64_t>(), w.existingMask, &dc->hashFail);
	}
	PairCtx P = pairCtx(w, cellSize);

	int32_t runMax = w.runCount;
	w.runPairCount.ensure((size_t)(runMax + 1) * sizeof(uint32_t));
	w.runPairOffs.ensure((size_t)(runMax + 1) * sizeof(uint32_t));
	if (runMax > 0)
	{
		M3G_LAUNCH(kRunPairs<false>, blocksFor(runMax, 128), 128, s, P, w.activeKeys.as<uint64_t>(),
				   w.activeVals.as<uint32_t>(), w.runStarts.as<int32_t>(), runMax, &dc->runs,
				   w.stableKeys.as<uint64_t>(), w.stableVals.as<uint32_t>(), w.stableEntries,
				   w.runPairCount.as<uint32_t>(), nullptr, nullptr);
	}
	if (w.batched)
	{
		scanExclusive(w.runPairCount.as<uint32_t>(), w.runPairOffs.as<uint32_t>(), runMax, &dc->gridPairs, w.prim, s);
		w.overTotal = launchOverPairsBatch(w, P);
		return;
	}
	int64_t overTotal;
	OverCtx O = overCtx(w, n, &overTotal);
	w.overTotal = overTotal;
	w.overFlag.ensure((size_t)(overTotal + 1) * sizeof(uint32_t));
	w.overScan.ensure((size_t)(overTotal + 1) * sizeof(uint32_t));
	w.overKeys.ensure((size_t)(overTotal + 1) * sizeof(uint64_t));
	if (overTotal > 0)
	{
		M3G_LAUNCH(kOverPairs, blocksFor(overTotal, 256), 256, s, P, O, overTotal, w.overFlag.as<uint32_t>(),
				   w.overKeys.as<uint64_t>());
	}
	// the run-pair offsets and the oversized-candidate offsets do not depend on
	// one another: one launch
	scanExclusive2(w.runPairCount.as<uint32_t>(), w.runPairOffs.as<uint32_t>(), runMax, &dc->gridPairs,
				   w.overFlag.as<uint32_t>(), w.overScan.as<uint32_t>(), overTotal, &dc->overPairs, w.prim, s);
}

// After the second sync: write the admitted pairs in emission order, keep the
// first occurrence of each, compact.  The count of new contacts stays on the
// device; the host only knows its upper bound (all admitted pairs).
void launchPairEmit(DevWorld& w, int32_t n, float cellSize)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	PairCtx P = pairCtx(w, cellSize);
	int32_t runMax = w.runCount;
	int64_t gridPairs = w.hostCounters->gridPairs;
	int64_t overPairs = w.hostCounters->overPairs;
	int64_t total = gridPairs + overPairs;
	w.pairTotal = total;
	w.pairKeys.ensure((size_t)(total + 1) * sizeof(uint64_t));
	uint64_t* pk = w.pairKeys.as<uint64_t>();
	if (runMax > 0 && gridPairs > 0)
	{
		M3G_LAUNCH(kRunPairs<true>, blocksFor(runMax, 128), 128, s, P, w.activeKeys.as<uint64_t>(),
				   w.activeVals.as<uint32_t>(), w.runStarts.as<int32_t>(), runMax, &dc->runs,
				   w.stableKeys.as<uint64_t>(), w.stableVals.as<uint32_t>(), w.stableEntries, nullptr,
				   w.runPairOffs.as<uint32_t>(), pk);
	}
	const int64_t overTotal = w.overTotal;
	if (overPairs > 0)
	{
		M3G_LAUNCH(kScatterKeys, blocksFor(overTotal, 256), 256, s, w.overFlag.as<uint32_t>(),
				   w.overScan.as<uint32_t>(), w.overKeys.as<uint64_t>(), overTotal, pk + gridPairs);
	}

	uint32_t ncap = tableCapacity(total);
	w.newSet.ensure((size_t)ncap * sizeof(uint64_t));
	w.newSetPos.ensure((size_t)ncap * sizeof(uint32_t));
	w.newMask = ncap - 1;
	w.keepFlag.ensure((size_t)(total + 1) * sizeof(uint32_t));
	w.keepScan.ensure((size_t)(total + 1) * sizeof(uint32_t));
	w.newContactKeys.ensure((size_t)(total + 1) * sizeof(uint64_t));
	if (total > 0)
	{
		fillWords2(w.newSet.ptr, 0xFFFFFFFFu, (size_t)ncap * sizeof(uint64_t), w.newSetPos.ptr, 0xFFFFFFFFu,
				   (size_t)ncap * sizeof(uint32_t), s);
		M3G_LAUNCH(kDedupeMark, blocksFor(total, 256), 256, s, pk, total, w.newSet.as<uint64_t>(),
				   w.newSetPos.as<uint32_t>(), w.newMask, &dc->hashFail);
		M3G_LAUNCH(kDedupeKeep, blocksFor(total, 256), 256, s, pk, total, w.newSet.as<uint64_t>(),
				   w.newSetPos.as<uint32_t>(), w.newMask, w.keepFlag.as<uint32_t>());
	}
	scanExclusive(w.keepFlag.as<uint32_t>(), w.keepScan.as<uint32_t>(), total, &dc->newContacts, w.prim, s);
	if (total > 0)
	{
		M3G_LAUNCH(kScatterKeys, blocksFor(total, 256), 256, s, w.keepFlag.as<uint32_t>(), w.keepScan.as<uint32_t>(), pk,
				   total, w.newContactKeys.as<uint64_t>());
	}
}

// ---------------------------------------------------------------------------
// contact creation (reference src/world.cpp:1540-1568)
// ---------------------------------------------------------------------------

__global__ void kCreateContacts(BodySoA B, ContactSoA C, const uint64_t* keys, int32_t maxCount,
								const uint32_t* newCount, int32_t base, uint32_t* contactCountDev)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	uint32_t count = *newCount;
	if (k == 0)
	{
		*contactCountDev = (uint32_t)base + count;
	}
	if (k >= maxCount || k >= (int)count)
	{
		return;
	}
	int c = base + k;
	uint64_t key = keys[k];
	int32_t lo = (int32_t)(key >> 32), hi = (int32_t)(uint32_t)key;
	const BodyCold& a = B.cold[lo];
	const BodyCold& b = B.cold[hi];
	C.bodies[c] = make_int2(lo, hi);
	C.pointCount[c] = 0;
	bool sensor = ((B.state[lo] | B.state[hi]) & kStSensor) != 0;
	bool curved = a.shape.type != kBox || b.shape.type != kBox;
	C.flags[c] = (uint8_t)((sensor ? kCFSensor : 0) | (curved ? kCFCurved : 0));
	C.normal[c] = make_float4(0.0f, 1.0f, 0.0f, sqrtf(a.friction * b.friction));
	C.mat[c] = make_float2(a.restitution > b.restitution ? a.restitution : b.restitution,
						   sqrtf(a.rollingResistance * b.rollingResistance));
	float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	C.cachePosA[c] = z;
	C.cacheRotA[c] = z;
	C.cachePosB[c] = z;
	C.cacheRotB[c] = z;
	for (int s = 0; s < 4; ++s)
	{
		size_t p = pidx(C, c, s);
		C.pAnchorA[p] = z;
		C.pAnchorB[p] = z;
		C.pFricA[p] = z;
		C.pFricB[p] = z;
		C.pSlip[p] = z;
		C.pRA[p] = z;
		C.pRB[p] = z;
		C.pJA[p] = z;
		C.pJB[p] = z;
	}
}

// Appends the new contacts after the w.contactCount existing ones; the new
// count is written to the device counter, the host keeps the upper bound.
void launchCreateContacts(DevWorld& w)
{
	StepCounters* dc = devCounters(w);
	int32_t maxNew = (int32_t)w.pairTotal;
	M3G_LAUNCH(kCreateContacts, blocksFor(maxNew > 0 ? maxNew : 1, 128), 128, w.stream, w.B, w.C,
			   w.newContactKeys.as<uint64_t>(), maxNew, &dc->newContacts, w.contactCount, &dc->contactCount);
	w.contactMax = w.contactCount + maxNew;
}

// ---------------------------------------------------------------------------
// removal of separated pairs: closed form of the reference's descending
// swap-remove (src/world.cpp:100-119, 1705-1735).  The reference visits the
// removed indices from the highest down; the k-th one it visits receives the
// element then at position count-k, which is either an original survivor or
// an element an earlier (higher) removal already moved there.  With
// S = count - removed and scan = number of removed indices below a position,
// count-k equals S + scan[i] for a removed i, so a hole i < S receives
//     p = S + scan[i];  while (removed[p]) p = S + scan[p];
// (each step follows an earlier move; the chain ends at a survivor at or above
// S).  Sources are distinct survivors >= S and destinations holes < S, so all
// holes are filled in parallel.  End events go out in descending index order.
// ---------------------------------------------------------------------------

__global__ void kRemovalFlags(BodySoA B, ContactSoA C, int32_t maxCount, const uint32_t* countDev, uint32_t* removeFlag,
							  uint32_t* evFlag)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c > maxCount)
	{
		return;
	}
	if (c >= (int)*countDev)
	{
		removeFlag[c] = 0;
		if (c < maxCount)
		{
			evFlag[c] = 0;
		}
		return;
	}
	int2 ab = C.bodies[c];
	uint32_t rm = 0;
	if ((B.bFlags[ab.x] & kBFAwake) || (B.bFlags[ab.y] & kBFAwake))
	{
		if (!overlap(loadFat(B, ab.x), loadFat(B, ab.y)))
		{
			rm = 1;
		}
	}
	removeFlag[c] = rm;
	evFlag[c] = (rm && (C.flags[c] & kCFTouching)) ? 1u : 0u;
}

__global__ void kRemovalEvents(const ContactSoA C, int32_t maxCount, const uint32_t* evFlag, const uint32_t* evScan,
							   const uint32_t* evTotal, int4* events)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= maxCount || !evFlag[c])
	{
		return;
	}
	uint32_t t = *evTotal;
	int2 ab = C.bodies[c];
	events[t - 1 - evScan[c]] = make_int4(ab.x, ab.y, (C.flags[c] & kCFSensor) ? 1 : 0, 0);
}

__device__ void copyContact(const ContactSoA& C, int dst, int src)
{
	C.bodies[dst] = C.bodies[src];
	C.pointCount[dst] = C.pointCount[src];
	C.flags[dst] = C.flags[src];
	C.normal[dst] = C.normal[src];
	C.mat[dst] = C.mat[src];
	C.cachePosA[dst] = C.cachePosA[src];
	C.cacheRotA[dst] = C.cacheRotA[src];
	C.cachePosB[dst] = C.cachePosB[src];
	C.cacheRotB[dst] = C.cacheRotB[src];
	for (int s = 0; s < 4; ++s)
	{
		size_t d = pidx(C, dst, s), o = pidx(C, src, s);
		C.pAnchorA[d] = C.pAnchorA[o];
		C.pAnchorB[d] = C.pAnchorB[o];
		C.pFricA[d] = C.pFricA[o];
		C.pFricB[d] = C.pFricB[o];
		C.pSlip[d] = C.pSlip[o];
		C.pRA[d] = C.pRA[o];
		C.pRB[d] = C.pRB[o];
		C.pJA[d] = C.pJA[o];
		C.pJB[d] = C.pJB[o];
	}
}

__global__ void kRemovalMoves(ContactSoA C, int32_t maxCount, const uint32_t* countDev, const uint32_t* removedDev,
							  const uint32_t* removeFlag, const uint32_t* removeScan)
{
	M3G_KERNEL_BEGIN();
	int32_t count = (int32_t)*countDev;
	int32_t S = count - (int32_t)*removedDev;
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= S || i >= maxCount || !removeFlag[i])
	{
		return;
	}
	int32_t p = S + (int32_t)removeScan[i];
	for (int guard = 0; guard <= count && p < count && removeFlag[p]; ++guard)
	{
		p = S + (int32_t)removeScan[p];
	}
	copyContact(C, i, p);
}

__global__ void kContactMoves(ContactSoA C, const int2* moves, int32_t count)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < count)
	{
		copyContact(C, moves[k].x, moves[k].y);
	}
}

// Sources of destroy-time moves all lie at or above the new contact count and
// destinations below it, so the moves are independent.
void launchContactMoves(DevWorld& w, const int2* hostMoves, int32_t count)
{
	if (count <= 0)
	{
		return;
	}
	w.moveSrc.ensure(sizeof(int2) * (size_t)count);
	cudaMemcpyAsync(w.moveSrc.ptr, hostMoves, sizeof(int2) * (size_t)count, cudaMemcpyHostToDevice, w.stream);
	// a copy from pageable memory returns once the source is staged, so the
	// caller may free hostMoves on return without waiting for the kernel
	M3G_LAUNCH(kContactMoves, blocksFor(count, 128), 128, w.stream, w.C, (const int2*)w.moveSrc.ptr, count);
}

__global__ void kContactAdjCount(const int2* bodies, int32_t count, uint32_t* perBody)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < count)
	{
		int2 ab = bodies[i];
		atomicAdd(&perBody[ab.x], 1u);
		atomicAdd(&perBody[ab.y], 1u);
	}
}

__global__ void kContactAdjFill(const int2* bodies, int32_t count, const uint32_t* start, uint32_t* cursor,
								int32_t* list)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < count)
	{
		int2 ab = bodies[i];
		list[start[ab.x] + atomicAdd(&cursor[ab.x], 1u)] = i;
		list[start[ab.y] + atomicAdd(&cursor[ab.y], 1u)] = i;
	}
}

// Per-body contact lists of the current contact array (CSR: adjStart has
// bodies + 1 offsets, adjList 2 x contacts indices).  The order inside one
// body's list is not fixed (atomic slots); its user sorts them.  Runs on
// stream s with the scan scratch prim (the world's own, or a second one when
// s is not the world's stream).
void launchContactAdjacency(DevWorld& w, int32_t bodies, cudaStream_t s, PrimScratch& prim)
{
	int32_t c = w.contactCount;
	size_t n4 = (size_t)(bodies + 1) * sizeof(uint32_t);
	w.adjCount.ensure(n4);
	w.adjStart.ensure(n4);
	w.adjList.ensure((size_t)(2 * (size_t)c + 1) * sizeof(int32_t));
	cudaMemsetAsync(w.adjCount.ptr, 0, n4, s);
	if (c > 0)
	{
		M3G_LAUNCH(kContactAdjCount, blocksFor(c, 256), 256, s, (const int2*)w.C.bodies, c,
				   w.adjCount.as<uint32_t>());
	}
	scanExclusive(w.adjCount.as<uint32_t>(), w.adjStart.as<uint32_t>(), bodies + 1, nullptr, prim, s);
	if (c > 0)
	{
		cudaMemsetAsync(w.adjCount.ptr, 0, n4, s);
		M3G_LAUNCH(kContactAdjFill, blocksFor(c, 256), 256, s, (const int2*)w.C.bodies, c, w.adjStart.as<uint32_t>(),
				   w.adjCount.as<uint32_t>(), w.adjList.as<int32_t>());
	}
}

__global__ void kRemovalFinish(uint32_t* countDev, const uint32_t* removedDev)
{
	M3G_KERNEL_BEGIN();
	*countDev -= *removedDev;
}

void launchRemoval(DevWorld& w)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	int32_t M = w.contactMax; // upper bound of the device count
	size_t c4 = (size_t)(M + 2) * sizeof(uint32_t);
	w.removeFlag.ensure(c4);
	w.removeScan.ensure(c4);
	w.evEndFlag.ensure(c4);
	w.evBeginFlag.ensure(c4);
	w.evRemoval.ensure((size_t)(M + 1) * sizeof(int4));
	w.moveSrc.ensure(c4);
	M3G_LAUNCH(kRemovalFlags, blocksFor(M + 1, 256), 256, s, w.B, w.C, M, &dc->contactCount, w.removeFlag.as<uint32_t>(),
			   w.evEndFlag.as<uint32_t>());
	// M + 1 entries so that removeScan[count] exists
	scanExclusive2(w.removeFlag.as<uint32_t>(), w.removeScan.as<uint32_t>(), M + 1, &dc->removed,
				   w.evEndFlag.as<uint32_t>(), w.evBeginFlag.as<uint32_t>(), M, &dc->endRemoval, w.prim, s);
	if (M > 0)
	{
		M3G_LAUNCH(kRemovalEvents, blocksFor(M, 256), 256, s, w.C, M, w.evEndFlag.as<uint32_t>(),
				   w.evBeginFlag.as<uint32_t>(), &dc->endRemoval, w.evRemoval.as<int4>());
		M3G_LAUNCH(kRemovalMoves, blocksFor(M, 256), 256, s, w.C, M, &dc->contactCount, &dc->removed,
				   w.removeFlag.as<uint32_t>(), w.removeScan.as<uint32_t>());
	}
	M3G_LAUNCH(kRemovalFinish, 1, 1, s, &dc->contactCount, &dc->removed);
}

} // namespace m3g

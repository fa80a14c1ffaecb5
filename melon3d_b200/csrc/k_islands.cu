// Islands, sleep and the end of the step.
//
// Islands: union-find over touching non-sensor dynamic-dynamic contacts and
// dynamic-dynamic joints, with the larger root always hooked under the
// smaller one, so every component's root is its smallest body index - the
// same canonical label the reference's serial union-find produces.  Awake
// islands wake all their bodies.  Contacts (and joints) of each island keep
// the reference's ascending index order - the Gauss-Seidel and colouring
// order - through a stable radix sort on the label.  Bodies are grouped by
// counting; their order inside an island is free, because every per-body
// stage (integration, reconstruction, colour-mask reset, sleep timers) is
// independent of the other bodies.
//
// Every count stays on the device: kernels are bounded by host-side upper
// bounds and read the exact counts from StepCounters, and the whole stage is
// skipped on the device when no dynamic body is awake (the reference's
// early-out).  (reference src/world.cpp:1848-2010, 2060-2166)
#include "m3d_dev.cuh"

#include <float.h>

namespace m3g
{

__global__ void kAnyAwakeDynamic(const uint8_t* bFlags, int32_t n, uint32_t* flag)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && (bFlags[i] & (kBFDynamic | kBFAwake)) == (kBFDynamic | kBFAwake))
	{
		*flag = 1;
	}
}

// the flag starts at zero: the step's counters are reset at its start
void launchAnyAwakeDynamic(DevWorld& w, int32_t n)
{
	StepCounters* dc = devCounters(w);
	if (n > 0)
	{
		M3G_LAUNCH(kAnyAwakeDynamic, blocksFor(n, 256), 256, w.stream, w.B.bFlags, n, &dc->anyAwakeDynamic);
	}
}

__global__ void kInitParent(int32_t* parent, int32_t n, const uint32_t* active, uint32_t* labelCount,
							uint32_t* cursor)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		// counts are cleared even when nothing is awake, so every later stage
		// sees zero islands; the labels of the last build are kept
		labelCount[i] = 0;
		cursor[i] = 0;
		if (*active)
		{
			parent[i] = i;
		}
	}
}

__device__ __forceinline__ int32_t ufFind(int32_t* parent, int32_t x)
{
	volatile int32_t* p = parent;
	int32_t px = p[x];
	while (px != x)
	{
		int32_t gp = p[px];
		if (gp != px)
		{
			p[x] = gp; // path halving: gp is an ancestor of x
		}
		x = px;
		px = p[x];
	}
	return x;
}

// Root of x without writing: the labelling pass stores each body's root into
// the same array, and a halving write there could replace a label already
// written with an intermediate ancestor.
__device__ __forceinline__ int32_t ufRoot(const int32_t* parent, int32_t x)
{
	const volatile int32_t* p = parent;
	int32_t px = p[x];
	while (px != x)
	{
		x = px;
		px = p[x];
	}
	return x;
}

__device__ void ufUnite(int32_t* parent, int32_t a, int32_t b)
{
	for (;;)
	{
		a = ufFind(parent, a);
		b = ufFind(parent, b);
		if (a == b)
		{
			return;
		}
		if (a > b)
		{
			int32_t t = a;
			a = b;
			b = t;
		}
		int32_t old = atomicCAS(&parent[b], b, a);
		if (old == b)
		{
			return;
		}
	}
}

__global__ void kUnionContacts(const ContactSoA C, int32_t maxCount, const uint32_t* countDev, const uint8_t* bFlags,
							   int32_t* parent, const uint32_t* active)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= maxCount || c >= (int)*countDev || !*active)
	{
		return;
	}
	uint8_t fl = C.flags[c];
	if (!(fl & kCFTouching) || (fl & kCFSensor))
	{
		return;
	}
	int2 ab = C.bodies[c];
	if ((bFlags[ab.x] & kBFDynamic) && (bFlags[ab.y] & kBFDynamic))
	{
		ufUnite(parent, ab.x, ab.y);
	}
}

__global__ void kUnionJoints(const JointRec* joints, int32_t count, const BodyCold* cold, int32_t* parent,
							 const uint32_t* active)
{
	M3G_KERNEL_BEGIN();
	int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= count || !*active)
	{
		return;
	}
	const JointRec& jr = joints[j];
	if (jr.inUse && cold[jr.bodyA].type == kDynamic && cold[jr.bodyB].type == kDynamic)
	{
		ufUnite(parent, jr.bodyA, jr.bodyB);
	}
}

__global__ void kLabels(int32_t* parent, int32_t n, const uint8_t* bFlags, int32_t* label, uint32_t* islandFlag,
						uint32_t* islandCount, const uint32_t* active)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n || !*active)
	{
		return;
	}
	islandFlag[i] = 0;
	if (bFlags[i] & kBFDynamic)
	{
		// label and parent are one array: only roots are written here, which
		// keeps every value any thread can read an ancestor of its body
		int32_t r = ufRoot(parent, i);
		label[i] = r;
		if (r == i)
		{
			atomicAdd(islandCount, 1u);
		}
	}
	else
	{
		label[i] = -1;
	}
}

__global__ void kIslandAwake(const uint8_t* bFlags, int32_t n, const int32_t* label, uint32_t* islandFlag,
							 const uint32_t* active)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && *active && (bFlags[i] & kBFDynamic) && (bFlags[i] & kBFAwake))
	{
		islandFlag[label[i]] = 1;
	}
}

// wake every body of an awake island and count the island's bodies
__global__ void kIslandBodies(BodySoA B, int32_t n, const int32_t* label, const uint32_t* islandFlag,
							  uint32_t* labelCount, uint32_t* stableDirty, const uint32_t* active)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n || !*active)
	{
		return;
	}
	if ((B.bFlags[i] & kBFDynamic) && islandFlag[label[i]])
	{
		if (!(B.state[i] & kStAwake))
		{
			wakeBody(B, i, stableDirty);
		}
		atomicAdd(&labelCount[label[i]], 1u);
	}
}

__global__ void kIslandListFlags(const uint32_t* labelCount, int32_t n, uint32_t* flag)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		flag[i] = labelCount[i] > 0 ? 1u : 0u;
	}
}

__global__ void kIslandListCompact(const uint32_t* flag, const uint32_t* offs, int32_t n, int32_t* islandLabels)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && flag[i])
	{
		islandLabels[offs[i]] = i;
	}
}

__global__ void kPlaceBodies(const BodySoA B, int32_t n, const int32_t* label, const uint32_t* islandFlag,
							 const uint32_t* labelStart, uint32_t* cursor, uint32_t* bodyVals, const uint32_t* active)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n || !*active)
	{
		return;
	}
	if ((B.bFlags[i] & kBFDynamic) && islandFlag[label[i]])
	{
		int32_t l = label[i];
		uint32_t slot = atomicAdd(&cursor[l], 1u);
		bodyVals[labelStart[l] + slot] = (uint32_t)i;
	}
}

__global__ void kContactIslandFlags(const ContactSoA C, int32_t maxCount, const uint32_t* countDev,
									const uint8_t* bFlags, const int32_t* label, const uint32_t* islandFlag,
									uint32_t* flag, uint32_t* touchingCount, uint32_t* pointCount, const uint32_t* active)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	uint32_t f = 0, points = 0;
	if (c < maxCount && c < (int)*countDev && *active)
	{
		uint8_t fl = C.flags[c];
		if (fl & kCFTouching)
		{
			atomicAdd(touchingCount, 1u);
			if (!(fl & kCFSensor))
			{
				int2 ab = C.bodies[c];
				int32_t dyn = (bFlags[ab.x] & kBFDynamic) ? ab.x : ab.y;
				if ((bFlags[dyn] & kBFDynamic) && islandFlag[label[dyn]])
				{
					f = 1;
					points = (uint32_t)C.pointCount[c];
				}
			}
		}
	}
	if (c < maxCount)
	{
		flag[c] = f;
	}
	// warp total of the island points, one atomic per warp
	points = __reduce_add_sync(0xffffffffu, points);
	if ((threadIdx.x & 31) == 0 && points != 0)
	{
		atomicAdd(pointCount, points);
	}
}

__global__ void kJointIslandFlags(const JointRec* joints, int32_t count, const BodyCold* cold, const int32_t* label,
								  const uint32_t* islandFlag, uint32_t* flag, const uint32_t* active)
{
	M3G_KERNEL_BEGIN();
	int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= count)
	{
		return;
	}
	uint32_t f = 0;
	const JointRec& jr = joints[j];
	if (*active && jr.inUse)
	{
		int32_t dyn = cold[jr.bodyA].type == kDynamic ? jr.bodyA : jr.bodyB;
		if (cold[dyn].type == kDynamic && islandFlag[label[dyn]])
		{
			f = 1;
		}
	}
	flag[j] = f;
}

// (label, index) pairs of the flagged items, in index order
__global__ void kLabelPairs(const uint32_t* flag, const uint32_t* offs, int32_t count, const int32_t* label,
							const int2* contactBodies, const JointRec* joints, const uint8_t* bFlags, const BodyCold* cold,
							int mode, uint64_t* keys, uint32_t* vals)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count || !flag[i])
	{
		return;
	}
	int32_t dyn;
	if (mode == 1)
	{
		int2 ab = contactBodies[i];
		dyn = (bFlags[ab.x] & kBFDynamic) ? ab.x : ab.y;
	}
	else
	{
		const JointRec& jr = joints[i];
		dyn = cold[jr.bodyA].type == kDynamic ? jr.bodyA : jr.bodyB;
	}
	uint32_t o = offs[i];
	keys[o] = (uint64_t)(uint32_t)label[dyn];
	vals[o] = (uint32_t)i;
}

__device__ __forceinline__ int32_t lowerBound64(const uint64_t* keys, int32_t n, uint64_t k)
{
	int32_t lo = 0, hi = n;
	while (lo < hi)
	{
		int32_t mid = (lo + hi) >> 1;
		if (keys[mid] < k)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo;
}

__global__ void kIslandTable(const int32_t* islandLabels, int32_t maxIslands, const uint32_t* islandsDev,
							 const uint32_t* labelStart, const uint32_t* labelCount, const uint64_t* contactKeys,
							 const uint32_t* contactsDev, const uint64_t* jointKeys, const uint32_t* jointsDev,
							 IslandRec* islands, int32_t* coloredList, int32_t* serialList, int32_t* tinyList,
							 int32_t* giantList, int32_t giantContacts, int32_t tinyContacts, StepCounters* dc)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= maxIslands || k >= (int)*islandsDev)
	{
		return;
	}
	int32_t lab = islandLabels[k];
	uint64_t key = (uint64_t)(uint32_t)lab;
	int32_t nc = (int32_t)*contactsDev;
	int32_t nj = jointsDev != nullptr ? (int32_t)*jointsDev : 0;
	IslandRec r;
	r.label = lab;
	r.bodyStart = (int32_t)labelStart[lab];
	r.bodyCount = (int32_t)labelCount[lab];
	r.contactStart = lowerBound64(contactKeys, nc, key);
	r.contactCount = lowerBound64(contactKeys, nc, key + 1) - r.contactStart;
	r.jointStart = nj > 0 ? lowerBound64(jointKeys, nj, key) : 0;
	r.jointCount = nj > 0 ? lowerBound64(jointKeys, nj, key + 1) - r.jointStart : 0;
	if (r.contactCount >= giantContacts && r.contactCount >= kBigIslandContacts)
	{
		r.kind = 3;
		giantList[atomicAdd(&dc->giantIslands, 1u)] = k;
	}
	else if (r.contactCount >= kBigIslandContacts)
	{
		r.kind = 2;
		coloredList[atomicAdd(&dc->coloredIslands, 1u)] = k;
	}
	else if (r.contactCount > 0 || r.jointCount > 0)
	{
		r.kind = 1;
		atomicAdd(&dc->serialIslands, 1u);
		atomicAdd(&dc->serialBodies, (uint32_t)r.bodyCount);
		atomicAdd(&dc->serialContacts, (uint32_t)r.contactCount);
		if (r.contactCount <= tinyContacts && r.jointCount == 0)
		{
			tinyList[atomicAdd(&dc->tinyIslands, 1u)] = k;
			atomicAdd(&dc->tinyBodies, (uint32_t)r.bodyCount);
			atomicAdd(&dc->tinyContacts, (uint32_t)r.contactCount);
		}
		else
		{
			serialList[atomicAdd(&dc->warpIslands, 1u)] = k;
		}
	}
	else
	{
		r.kind = 0;
		atomicAdd(&dc->freeIslands, 1u);
	}
	islands[k] = r;
}

// sort key of a tiny island: contact count (up to 15, descending) above body
// count (up to 15, descending) above the shape of its first body (the
// collision code its thread runs)
__global__ void kTinyKeys(const IslandRec* islands, const int32_t* tinyList, int32_t maxN, const uint32_t* countDev,
						  const uint32_t* bodyVals, const BodyCold* cold, uint64_t* keys)
{
	M3G_KERNEL_BEGIN();
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= maxN || k >= (int)*countDev)
	{
		return;
	}
	const IslandRec r = islands[tinyList[k]];
	const uint32_t c = r.contactCount < 15 ? (uint32_t)r.contactCount : 15u;
	const uint32_t b = r.bodyCount < 15 ? (uint32_t)r.bodyCount : 15u;
	const uint32_t shape = (uint32_t)cold[bodyVals[r.bodyStart]].shape.type & 3u;
	keys[k] = (uint64_t)(((((15u - c) << 4) | (15u - b)) << 2) | shape); // largest islands first
}

// sort key of a warp island, largest first: 1023 minus its contacts plus
// twice its joints
__global__ void kWarpIslandKeys(const IslandRec* islands, const int32_t* serialList, int32_t maxN,
								const uint32_t* countDev, uint64_t* keys)
{
	M3G_KERNEL_BEGIN();
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= maxN || k >= (int)*countDev)
	{
		return;
	}
	const IslandRec r = islands[serialList[k]];
	const int32_t size = r.contactCount + 2 * r.jointCount;
	keys[k] = (uint64_t)(1023 - (size < 1023 ? size : 1023));
}

static int bitsFor(int64_t n)
{
	int b = 1;
	while (b < 63 && (1ll << b) <= n)
	{
		++b;
	}
	return b;
}

void launchIslands(DevWorld& w, int32_t n)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	const uint32_t* active = &dc->anyAwakeDynamic;
	int32_t M = w.contactMax;
	size_t n4 = (size_t)(n + 1) * sizeof(uint32_t);
	w.label.ensure(n4);
	w.islandFlag.ensure(n4);
	w.labelCount.ensure(n4);
	w.labelStart.ensure(n4);
	w.labelCursor.ensure(n4);
	w.islandListFlag.ensure(n4);
	w.islandListOffs.ensure(n4);
	w.islandLabels.ensure(n4);
	w.bodyVals.ensure(n4);
	w.islands.ensure((size_t)(n + 1) * sizeof(IslandRec));
	w.coloredList.ensure(n4);
	w.serialList.ensure(n4);
	w.tinyList.ensure(n4);
	w.giantList.ensure(n4);
	int32_t* parent = w.label.as<int32_t>();
	M3G_LAUNCH(kInitParent, blocksFor(n, 256), 256, s, parent, n, active, w.labelCount.as<uint32_t>(),
			   w.labelCursor.as<uint32_t>());
	if (M > 0)
	{
		M3G_LAUNCH(kUnionContacts, blocksFor(M, 256), 256, s, w.C, M, &dc->contactCount, w.B.bFlags, parent, active);
	}
	if (w.jointCount > 0)
	{
		M3G_LAUNCH(kUnionJoints, blocksFor(w.jointCount, 128), 128, s, w.joints.as<JointRec>(), w.jointCount, w.B.cold,
				   parent, active);
	}
	M3G_LAUNCH(kLabels, blocksFor(n, 256), 256, s, parent, n, w.B.bFlags, w.label.as<int32_t>(),
			   w.islandFlag.as<uint32_t>(), &dc->islandCount, active);
	M3G_LAUNCH(kIslandAwake, blocksFor(n, 256), 256, s, w.B.bFlags, n, w.label.as<int32_t>(), w.islandFlag.as<uint32_t>(),
			   active);
	M3G_LAUNCH(kIslandBodies, blocksFor(n, 256), 256, s, w.B, n, w.label.as<int32_t>(), w.islandFlag.as<uint32_t>(),
			   w.labelCount.as<uint32_t>(), stableDirtyWords(w), active);
	// bodies per island: label counts -> starts -> placement
	M3G_LAUNCH(kIslandListFlags, blocksFor(n, 256), 256, s, w.labelCount.as<uint32_t>(), n,
			   w.islandListFlag.as<uint32_t>());
	scanExclusive2(w.labelCount.as<uint32_t>(), w.labelStart.as<uint32_t>(), n, &dc->islandBodies,
				   w.islandListFlag.as<uint32_t>(), w.islandListOffs.as<uint32_t>(), n, &dc->awakeIslands, w.prim, s);
	M3G_LAUNCH(kIslandListCompact, blocksFor(n, 256), 256, s, w.islandListFlag.as<uint32_t>(),
			   w.islandListOffs.as<uint32_t>(), n, w.islandLabels.as<int32_t>());
	M3G_LAUNCH(kPlaceBodies, blocksFor(n, 256), 256, s, w.B, n, w.label.as<int32_t>(), w.islandFlag.as<uint32_t>(),
			   w.labelStart.as<uint32_t>(), w.labelCursor.as<uint32_t>(), w.bodyVals.as<uint32_t>(), active);

	// contacts per island, ascending contact index inside each island
	uint64_t labelMask = (1ull << bitsFor(n)) - 1ull;
	w.removeFlag.ensure((size_t)(M + 1) * sizeof(uint32_t));
	w.removeScan.ensure((size_t)(M + 1) * sizeof(uint32_t));
	w.contactKeys.ensure((size_t)(M + 1) * sizeof(uint64_t));
	w.contactVals.ensure((size_t)(M + 1) * sizeof(uint32_t));
	if (M > 0)
	{
		M3G_LAUNCH(kContactIslandFlags, blocksFor(M, 256), 256, s, w.C, M, &dc->contactCount, w.B.bFlags,
				   w.label.as<int32_t>(), w.islandFlag.as<uint32_t>(), w.removeFlag.as<uint32_t>(), &dc->touchingCount,
				   &dc->islandPoints, active);
	}
	scanExclusive(w.removeFlag.as<uint32_t>(), w.removeScan.as<uint32_t>(), M, &dc->islandContacts, w.prim, s);
	if (M > 0)
	{
		M3G_LAUNCH(kLabelPairs, blocksFor(M, 256), 256, s, w.removeFlag.as<uint32_t>(), w.removeScan.as<uint32_t>(), M,
				   w.label.as<int32_t>(), w.C.bodies, w.joints.as<JointRec>(), w.B.bFlags, w.B.cold, 1,
				   w.contactKeys.as<uint64_t>(), w.contactVals.as<uint32_t>());
		radixSortPairs(w.contactKeys.as<uint64_t>(), w.contactVals.as<uint32_t>(), M, labelMask, w.prim, s,
					   &dc->islandContacts);
	}
	// joints per island
	int32_t J = w.jointCount;
	if (J > 0)
	{
		w.overFlagS.ensure((size_t)(J + 1) * sizeof(uint32_t));
		w.jointScan.ensure((size_t)(J + 1) * sizeof(uint32_t));
		w.jointKeys.ensure((size_t)(J + 1) * sizeof(uint64_t));
		w.jointVals.ensure((size_t)(J + 1) * sizeof(uint32_t));
		M3G_LAUNCH(kJointIslandFlags, blocksFor(J, 128), 128, s, w.joints.as<JointRec>(), J, w.B.cold,
				   w.label.as<int32_t>(), w.islandFlag.as<uint32_t>(), w.overFlagS.as<uint32_t>(), active);
		scanExclusive(w.overFlagS.as<uint32_t>(), w.jointScan.as<uint32_t>(), J, &dc->islandJoints, w.prim, s);
		M3G_LAUNCH(kLabelPairs, blocksFor(J, 128), 128, s, w.overFlagS.as<uint32_t>(), w.jointScan.as<uint32_t>(), J,
				   w.label.as<int32_t>(), w.C.bodies, w.joints.as<JointRec>(), w.B.bFlags, w.B.cold, 2,
				   w.jointKeys.as<uint64_t>(), w.jointVals.as<uint32_t>());
		radixSortPairs(w.jointKeys.as<uint64_t>(), w.jointVals.as<uint32_t>(), J, labelMask, w.prim, s,
					   &dc->islandJoints);
	}
	M3G_LAUNCH(kIslandTable, blocksFor(n, 128), 128, s, w.islandLabels.as<int32_t>(), n, &dc->awakeIslands,
			   w.labelStart.as<uint32_t>(), w.labelCount.as<uint32_t>(), w.contactKeys.as<uint64_t>(),
			   &dc->islandContacts, w.jointKeys.as<uint64_t>(), J > 0 ? &dc->islandJoints : nullptr,
			   w.islands.as<IslandRec>(), w.coloredList.as<int32_t>(), w.serialList.as<int32_t>(),
			   w.tinyList.as<int32_t>(), w.giantList.as<int32_t>(), w.giantIslandContacts,
			   w.lastSerialIslands > w.tinyModeIslands ? w.tinyContacts : 0, dc);
	if (w.lastSerialIslands > w.tinyModeIslands && w.tinyContacts > 0)
	{
		// one thread per tiny island: group islands of equal contact and body
		// counts into the same warps (the list order, filled by atomics, is
		// arbitrary anyway, and every island is solved on its own)
		w.tinyKeys.ensure((size_t)(n + 1) * sizeof(uint64_t));
		M3G_LAUNCH(kTinyKeys, blocksFor(n, 256), 256, s, w.islands.as<IslandRec>(), w.tinyList.as<int32_t>(), n,
				   &dc->tinyIslands, w.bodyVals.as<uint32_t>(), w.B.cold, w.tinyKeys.as<uint64_t>());
		radixSortPairs(w.tinyKeys.as<uint64_t>(), (uint32_t*)w.tinyList.ptr, n, 0x3FFull, w.prim, s, &dc->tinyIslands);
		// the warp islands largest first, so the last wave of warps is not
		// left waiting on a few large islands
		M3G_LAUNCH(kWarpIslandKeys, blocksFor(n, 256), 256, s, w.islands.as<IslandRec>(), w.serialList.as<int32_t>(),
				   n, &dc->warpIslands, w.tinyKeys.as<uint64_t>());
		radixSortPairs(w.tinyKeys.as<uint64_t>(), (uint32_t*)w.serialList.ptr, n, 0x3FFull, w.prim, s,
					   &dc->warpIslands);
	}
	w.islandMax = n;
}

// ---------------------------------------------------------------------------
// sleep (reference src/world.cpp:2060-2108).  Per awake island, bodies are
// visited in ascending index order up to (not including) the first body with
// sleep disabled; the island sleeps when no such body exists and the
// smallest timer reached kTimeToSleep.
// ---------------------------------------------------------------------------

__global__ void kSleepInit(const int32_t* islandLabels, int32_t maxIslands, const uint32_t* islandsDev, int32_t* firstNo,
						   uint32_t* minBits)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < maxIslands && k < (int)*islandsDev)
	{
		int32_t lab = islandLabels[k];
		firstNo[lab] = 0x7FFFFFFF;
		minBits[lab] = __float_as_uint(FLT_MAX);
	}
}

__global__ void kSleepNoFlags(const BodySoA B, const uint32_t* vals, int32_t maxBodies, const uint32_t* bodiesDev,
							  const int32_t* label, int32_t* firstNo)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= maxBodies || k >= (int)*bodiesDev)
	{
		return;
	}
	int32_t i = (int32_t)vals[k];
	if (!(B.state[i] & kStEnableSleep))
	{
		atomicMin(&firstNo[label[i]], i);
	}
}

__global__ void kSleepUpdate(BodySoA B, const uint32_t* vals, int32_t maxBodies, const uint32_t* bodiesDev,
							 const int32_t* label, const int32_t* firstNo, uint32_t* minBits, float dt)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= maxBodies || k >= (int)*bodiesDev)
	{
		return;
	}
	int32_t i = (int32_t)vals[k];
	int32_t lab = label[i];
	if (i >= firstNo[lab])
	{
		return;
	}
	float energy = len2(ld3(B.vel[i])) + len2(ld3(B.angVel[i]));
	float2 sl = B.sleep[i];
	sl.y += kSleepEnergyAlpha * (energy - sl.y);
	if (sl.y > kSleepWakeFactor * kSleepEnergyThresh)
	{
		sl.x = 0.0f;
	}
	else if (sl.y < kSleepEnergyThresh)
	{
		sl.x += dt;
	}
	else
	{
		sl.x += 0.5f * dt;
	}
	B.sleep[i] = sl;
	atomicMin(&minBits[lab], __float_as_uint(sl.x));
}

__global__ void kSleepApply(BodySoA B, const uint32_t* vals, int32_t maxBodies, const uint32_t* bodiesDev,
							const int32_t* label, const int32_t* firstNo, const uint32_t* minBits,
							uint32_t* stableDirty, uint32_t* record, uint32_t* recordCount)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= maxBodies || k >= (int)*bodiesDev)
	{
		return;
	}
	int32_t i = (int32_t)vals[k];
	int32_t lab = label[i];
	if (firstNo[lab] != 0x7FFFFFFF || !(__uint_as_float(minBits[lab]) >= kTimeToSleep))
	{
		return;
	}
	B.state[i] &= (uint8_t)~kStAwake;
	float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	B.vel[i] = z;
	B.angVel[i] = z;
	B.bFlags[i] &= (uint8_t)~kBFAwake;
	stableDirty[worldOfBody(B, i)] = 1;
	if (record != nullptr)
	{
		record[atomicAdd(recordCount, 1u)] = (uint32_t)i;
	}
}

void launchSleep(DevWorld& w, float dt)
{
	StepCounters* dc = devCounters(w);
	int32_t nmax = w.islandMax;
	if (nmax <= 0)
	{
		return;
	}
	size_t cap = (size_t)w.bodyCap + 1;
	w.sleepFirstNo.ensure(cap * sizeof(int32_t));
	w.sleepMin.ensure(cap * sizeof(uint32_t));
	cudaStream_t s = w.stream;
	const uint32_t* vals = w.bodyVals.as<uint32_t>();
	const int32_t* lab = w.label.as<int32_t>();
	M3G_LAUNCH(kSleepInit, blocksFor(nmax, 256), 256, s, w.islandLabels.as<int32_t>(), nmax, &dc->awakeIslands,
			   w.sleepFirstNo.as<int32_t>(), w.sleepMin.as<uint32_t>());
	M3G_LAUNCH(kSleepNoFlags, blocksFor(nmax, 256), 256, s, w.B, vals, nmax, &dc->islandBodies, lab,
			   w.sleepFirstNo.as<int32_t>());
	M3G_LAUNCH(kSleepUpdate, blocksFor(nmax, 256), 256, s, w.B, vals, nmax, &dc->islandBodies, lab,
			   w.sleepFirstNo.as<int32_t>(), w.sleepMin.as<uint32_t>(), dt);
	M3G_LAUNCH(kSleepApply, blocksFor(nmax, 256), 256, s, w.B, vals, nmax, &dc->islandBodies, lab,
			   w.sleepFirstNo.as<int32_t>(), w.sleepMin.as<uint32_t>(), stableDirtyWords(w), w.sleepRecord,
			   &dc->sleptBodies);
}

// kinematic integration, one-step force clear, profile counters
// (reference src/world.cpp:2111-2155)
__global__ void kFinish(BodySoA B, int32_t n, float dt, int clearForces, StepCounters* dc)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	uint8_t f = B.bFlags[i];
	if ((f & kBFKinematic) && (f & kBFAwake))
	{
		V3 v = ld3(B.vel[i]);
		V3 w = ld3(B.angVel[i]);
		B.pos[i] = st3(madd(ld3(B.pos[i]), dt, v));
		B.rot[i] = stq(qintegrate(ldq(B.rot[i]), w, dt));
	}
	if (clearForces && (f & kBFDynamic))
	{
		float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		B.force[i] = z;
		B.torque[i] = z;
	}
	if (f & kBFInUse)
	{
		atomicAdd(&dc->bodyCount, 1u);
		if (f & kBFAwake)
		{
			atomicAdd(&dc->awakeBodyCount, 1u);
		}
	}
}

// the body counts start at zero: the step's counters are reset at its start
void launchFinish(DevWorld& w, int32_t n, float dt, bool clearForces)
{
	StepCounters* dc = devCounters(w);
	if (n > 0)
	{
		M3G_LAUNCH(kFinish, blocksFor(n, 256), 256, w.stream, w.B, n, dt, clearForces ? 1 : 0, dc);
	}
}

} // namespace m3g

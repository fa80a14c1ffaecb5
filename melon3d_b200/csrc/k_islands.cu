// Islands, sleep and the end of the step.
//
// Islands: union-find over touching non-sensor dynamic-dynamic contacts and
// dynamic-dynamic joints, with the larger root always hooked under the
// smaller one, so every component's root is its smallest body index - the
// same canonical label the reference's serial union-find produces.  Awake
// islands wake all their bodies; their contacts, joints and bodies are
// grouped per island by a stable sort on the label, which keeps the
// reference's ascending index order inside each island.
// (reference src/world.cpp:1848-2010, 2060-2166)
#include "m3d_dev.cuh"

#include <float.h>

namespace m3g
{

__global__ void kAnyAwakeDynamic(const uint8_t* bFlags, int32_t n, uint32_t* flag)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && (bFlags[i] & (kBFDynamic | kBFAwake)) == (kBFDynamic | kBFAwake))
	{
		*flag = 1;
	}
}

void launchAnyAwakeDynamic(DevWorld& w, int32_t n)
{
	StepCounters* dc = devCounters(w);
	cudaMemsetAsync(&dc->anyAwakeDynamic, 0, sizeof(uint32_t), w.stream);
	if (n > 0)
	{
		M3G_LAUNCH(kAnyAwakeDynamic, blocksFor(n, 256), 256, w.stream, w.B.bFlags, n, &dc->anyAwakeDynamic);
	}
}

__global__ void kInitParent(int32_t* parent, int32_t n)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		parent[i] = i;
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

__global__ void kUnionContacts(const ContactSoA C, int32_t count, const uint8_t* bFlags, int32_t* parent)
{
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= count)
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

__global__ void kUnionJoints(const JointRec* joints, int32_t count, const BodyCold* cold, int32_t* parent)
{
	int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= count)
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
						uint32_t* islandCount)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	islandFlag[i] = 0;
	if (bFlags[i] & kBFDynamic)
	{
		int32_t r = ufFind(parent, i);
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

__global__ void kIslandAwake(const uint8_t* bFlags, int32_t n, const int32_t* label, uint32_t* islandFlag)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && (bFlags[i] & kBFDynamic) && (bFlags[i] & kBFAwake))
	{
		islandFlag[label[i]] = 1;
	}
}

// wake every body of an awake island; flag the bodies to solve
__global__ void kIslandWakeBodies(BodySoA B, int32_t n, const int32_t* label, const uint32_t* islandFlag,
								  uint32_t* bodyFlag, uint32_t* stableDirty)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	uint32_t f = 0;
	if ((B.bFlags[i] & kBFDynamic) && islandFlag[label[i]])
	{
		f = 1;
		if (!(B.state[i] & kStAwake))
		{
			wakeBody(B, i, stableDirty);
		}
	}
	bodyFlag[i] = f;
}

__global__ void kContactIslandFlags(const ContactSoA C, int32_t count, const uint8_t* bFlags, const int32_t* label,
									const uint32_t* islandFlag, uint32_t* flag, uint32_t* touchingCount)
{
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= count)
	{
		return;
	}
	uint8_t fl = C.flags[c];
	uint32_t f = 0;
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
			}
		}
	}
	flag[c] = f;
}

__global__ void kJointIslandFlags(const JointRec* joints, int32_t count, const BodyCold* cold, const int32_t* label,
								  const uint32_t* islandFlag, uint32_t* flag)
{
	int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= count)
	{
		return;
	}
	const JointRec& jr = joints[j];
	uint32_t f = 0;
	if (jr.inUse)
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
__global__ void kLabelPairs(const uint32_t* flag, const uint32_t* offs, int32_t count, const int32_t* itemLabelOf,
							const int2* contactBodies, const JointRec* joints, const uint8_t* bFlags, const BodyCold* cold,
							int mode, uint64_t* keys, uint32_t* vals)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count || !flag[i])
	{
		return;
	}
	int32_t lab;
	if (mode == 0)
	{
		lab = itemLabelOf[i]; // bodies
	}
	else if (mode == 1)
	{
		int2 ab = contactBodies[i];
		int32_t dyn = (bFlags[ab.x] & kBFDynamic) ? ab.x : ab.y;
		lab = itemLabelOf[dyn];
	}
	else
	{
		const JointRec& jr = joints[i];
		int32_t dyn = cold[jr.bodyA].type == kDynamic ? jr.bodyA : jr.bodyB;
		lab = itemLabelOf[dyn];
	}
	uint32_t o = offs[i];
	keys[o] = (uint64_t)(uint32_t)lab;
	vals[o] = (uint32_t)i;
}

__global__ void kIslandStarts(const uint64_t* keys, int32_t n, uint32_t* flag)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
	}
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

__global__ void kIslandTable(const uint64_t* bodyKeys, int32_t nBodies, const uint32_t* startFlag,
							 const uint32_t* startOffs, const uint64_t* contactKeys, int32_t nContacts,
							 const uint64_t* jointKeys, int32_t nJoints, IslandRec* islands, int32_t nIslands,
							 StepCounters* dc)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nBodies || !startFlag[i])
	{
		return;
	}
	int32_t k = (int32_t)startOffs[i];
	uint64_t key = bodyKeys[i];
	int32_t end = i + 1;
	while (end < nBodies && bodyKeys[end] == key)
	{
		++end;
	}
	IslandRec r;
	r.label = (int32_t)key;
	r.bodyStart = i;
	r.bodyCount = end - i;
	r.contactStart = lowerBound64(contactKeys, nContacts, key);
	r.contactCount = lowerBound64(contactKeys, nContacts, key + 1) - r.contactStart;
	r.jointStart = lowerBound64(jointKeys, nJoints, key);
	r.jointCount = lowerBound64(jointKeys, nJoints, key + 1) - r.jointStart;
	if (r.contactCount >= kBigIslandContacts)
	{
		r.kind = 2;
		atomicAdd(&dc->coloredIslands, 1u);
	}
	else if (r.contactCount > 0 || r.jointCount > 0)
	{
		r.kind = 1;
		atomicAdd(&dc->serialIslands, 1u);
	}
	else
	{
		r.kind = 0;
		atomicAdd(&dc->freeIslands, 1u);
	}
	islands[k] = r;
	(void)nIslands;
}

// flag scan + (label, index) pairs + stable sort by label
static int32_t groupByLabel(DevWorld& w, int mode, int32_t count, DevBuf& flag, DevBuf& keys, DevBuf& vals,
							uint32_t* totalDev, uint32_t* totalHost)
{
	DevBuf& offs = w.removeScan;
	offs.ensure((size_t)(count + 1) * sizeof(uint32_t));
	scanExclusive(flag.as<uint32_t>(), offs.as<uint32_t>(), count, totalDev, w.prim, w.stream);
	readCounters(w);
	int32_t total = (int32_t)*totalHost;
	keys.ensure((size_t)(total + 1) * sizeof(uint64_t));
	vals.ensure((size_t)(total + 1) * sizeof(uint32_t));
	if (count > 0)
	{
		M3G_LAUNCH(kLabelPairs, blocksFor(count, 256), 256, w.stream, 
			flag.as<uint32_t>(), offs.as<uint32_t>(), count, w.label.as<int32_t>(), w.C.bodies,
			w.joints.as<JointRec>(), w.B.bFlags, w.B.cold, mode, keys.as<uint64_t>(), vals.as<uint32_t>());
	}
	if (total > 1)
	{
		reduceKeyRange(keys.as<uint64_t>(), total, w.prim, w.stream);
		cudaStreamSynchronize(w.stream);
		radixSortPairs(keys.as<uint64_t>(), vals.as<uint32_t>(), total, w.prim.hostReduce[0] ^ w.prim.hostReduce[1],
					   w.prim, w.stream);
	}
	return total;
}

void launchIslands(DevWorld& w, int32_t n)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	size_t n4 = (size_t)(n + 1) * sizeof(uint32_t);
	w.label.ensure(n4);
	w.islandFlag.ensure(n4);
	w.cellCountA.ensure(n4); // reused: per-body solve flag
	int32_t* parent = w.label.as<int32_t>();
	M3G_LAUNCH(kInitParent, blocksFor(n, 256), 256, s, parent, n);
	if (w.contactCount > 0)
	{
		M3G_LAUNCH(kUnionContacts, blocksFor(w.contactCount, 256), 256, s, w.C, w.contactCount, w.B.bFlags, parent);
	}
	if (w.jointCount > 0)
	{
		M3G_LAUNCH(kUnionJoints, blocksFor(w.jointCount, 128), 128, s, w.joints.as<JointRec>(), w.jointCount, w.B.cold,
																   parent);
	}
	cudaMemsetAsync(&dc->islandCount, 0, sizeof(uint32_t), s);
	cudaMemsetAsync(&dc->touchingCount, 0, sizeof(uint32_t), s);
	cudaMemsetAsync(&dc->coloredIslands, 0, 3 * sizeof(uint32_t), s);
	M3G_LAUNCH(kLabels, blocksFor(n, 256), 256, s, parent, n, w.B.bFlags, w.label.as<int32_t>(), w.islandFlag.as<uint32_t>(),
											  &dc->islandCount);
	M3G_LAUNCH(kIslandAwake, blocksFor(n, 256), 256, s, w.B.bFlags, n, w.label.as<int32_t>(), w.islandFlag.as<uint32_t>());
	M3G_LAUNCH(kIslandWakeBodies, blocksFor(n, 256), 256, s, w.B, n, w.label.as<int32_t>(), w.islandFlag.as<uint32_t>(),
														 w.cellCountA.as<uint32_t>(), &dc->stableDirty);
	int32_t cc = w.contactCount;
	w.removeFlag.ensure((size_t)(cc + 1) * sizeof(uint32_t));
	if (cc > 0)
	{
		M3G_LAUNCH(kContactIslandFlags, blocksFor(cc, 256), 256, s, w.C, cc, w.B.bFlags, w.label.as<int32_t>(),
																 w.islandFlag.as<uint32_t>(), w.removeFlag.as<uint32_t>(),
																 &dc->touchingCount);
	}
	w.overFlagS.ensure((size_t)(w.jointCount + 1) * sizeof(uint32_t));
	if (w.jointCount > 0)
	{
		M3G_LAUNCH(kJointIslandFlags, blocksFor(w.jointCount, 128), 128, s, w.joints.as<JointRec>(), w.jointCount, w.B.cold,
																		w.label.as<int32_t>(),
																		w.islandFlag.as<uint32_t>(),
																		w.overFlagS.as<uint32_t>());
	}

	int32_t nb = groupByLabel(w, 0, n, w.cellCountA, w.bodyKeys, w.bodyVals, &dc->islandBodies,
							  &w.hostCounters->islandBodies);
	int32_t nc = groupByLabel(w, 1, cc, w.removeFlag, w.contactKeys, w.contactVals, &dc->islandContacts,
							  &w.hostCounters->islandContacts);
	int32_t nj = groupByLabel(w, 2, w.jointCount, w.overFlagS, w.jointKeys, w.jointVals, &dc->islandJoints,
							  &w.hostCounters->islandJoints);

	// island table
	w.islandStartFlag.ensure((size_t)(nb + 1) * sizeof(uint32_t));
	w.runPairCount.ensure((size_t)(nb + 1) * sizeof(uint32_t));
	if (nb > 0)
	{
		M3G_LAUNCH(kIslandStarts, blocksFor(nb, 256), 256, s, w.bodyKeys.as<uint64_t>(), nb,
														  w.islandStartFlag.as<uint32_t>());
	}
	scanExclusive(w.islandStartFlag.as<uint32_t>(), w.runPairCount.as<uint32_t>(), nb, &dc->awakeIslands, w.prim, s);
	readCounters(w);
	int32_t ni = (int32_t)w.hostCounters->awakeIslands;
	w.islands.ensure((size_t)(ni + 1) * sizeof(IslandRec));
	if (nb > 0)
	{
		M3G_LAUNCH(kIslandTable, blocksFor(nb, 256), 256, s, 
			w.bodyKeys.as<uint64_t>(), nb, w.islandStartFlag.as<uint32_t>(), w.runPairCount.as<uint32_t>(),
			w.contactKeys.as<uint64_t>(), nc, w.jointKeys.as<uint64_t>(), nj, w.islands.as<IslandRec>(), ni, dc);
	}
	w.islandCount = ni;
	w.islandsBuiltFor = n;
	readCounters(w);
}

// ---------------------------------------------------------------------------
// sleep (reference src/world.cpp:2060-2108).  Per awake island, bodies are
// visited in ascending index order up to (not including) the first body with
// sleep disabled; the island sleeps when no such body exists and the
// smallest timer reached kTimeToSleep.
// ---------------------------------------------------------------------------

__global__ void kSleepInit(const IslandRec* islands, int32_t ni, int32_t* firstNo, uint32_t* minBits)
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < ni)
	{
		int32_t lab = islands[k].label;
		firstNo[lab] = 0x7FFFFFFF;
		minBits[lab] = __float_as_uint(FLT_MAX);
	}
}

__global__ void kSleepNoFlags(const BodySoA B, const uint64_t* keys, const uint32_t* vals, int32_t nb, int32_t* firstNo)
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nb)
	{
		return;
	}
	int32_t i = (int32_t)vals[k];
	if (!(B.state[i] & kStEnableSleep))
	{
		atomicMin(&firstNo[(int32_t)keys[k]], i);
	}
}

__global__ void kSleepUpdate(BodySoA B, const uint64_t* keys, const uint32_t* vals, int32_t nb, const int32_t* firstNo,
							 uint32_t* minBits, float dt)
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nb)
	{
		return;
	}
	int32_t i = (int32_t)vals[k];
	int32_t lab = (int32_t)keys[k];
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

__global__ void kSleepApply(BodySoA B, const uint64_t* keys, const uint32_t* vals, int32_t nb, const int32_t* firstNo,
							const uint32_t* minBits, uint32_t* stableDirty)
{
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= nb)
	{
		return;
	}
	int32_t lab = (int32_t)keys[k];
	if (firstNo[lab] != 0x7FFFFFFF || !(__uint_as_float(minBits[lab]) >= kTimeToSleep))
	{
		return;
	}
	int32_t i = (int32_t)vals[k];
	B.state[i] &= (uint8_t)~kStAwake;
	float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	B.vel[i] = z;
	B.angVel[i] = z;
	B.bFlags[i] &= (uint8_t)~kBFAwake;
	*stableDirty = 1;
}

void launchSleep(DevWorld& w, float dt)
{
	StepCounters* dc = devCounters(w);
	int32_t ni = w.islandCount;
	int32_t nb = (int32_t)w.hostCounters->islandBodies;
	if (ni <= 0 || nb <= 0)
	{
		return;
	}
	size_t cap = (size_t)w.bodyCap + 1;
	w.sleepFirstNo.ensure(cap * sizeof(int32_t));
	w.sleepMin.ensure(cap * sizeof(uint32_t));
	cudaStream_t s = w.stream;
	M3G_LAUNCH(kSleepInit, blocksFor(ni, 256), 256, s, w.islands.as<IslandRec>(), ni, w.sleepFirstNo.as<int32_t>(),
												   w.sleepMin.as<uint32_t>());
	M3G_LAUNCH(kSleepNoFlags, blocksFor(nb, 256), 256, s, w.B, w.bodyKeys.as<uint64_t>(), w.bodyVals.as<uint32_t>(), nb,
													  w.sleepFirstNo.as<int32_t>());
	M3G_LAUNCH(kSleepUpdate, blocksFor(nb, 256), 256, s, w.B, w.bodyKeys.as<uint64_t>(), w.bodyVals.as<uint32_t>(), nb,
													 w.sleepFirstNo.as<int32_t>(), w.sleepMin.as<uint32_t>(), dt);
	M3G_LAUNCH(kSleepApply, blocksFor(nb, 256), 256, s, w.B, w.bodyKeys.as<uint64_t>(), w.bodyVals.as<uint32_t>(), nb,
													w.sleepFirstNo.as<int32_t>(), w.sleepMin.as<uint32_t>(),
													&dc->stableDirty);
}

// kinematic integration, one-step force clear, profile counters
// (reference src/world.cpp:2111-2155)
__global__ void kFinish(BodySoA B, int32_t n, float dt, int clearForces, StepCounters* dc)
{
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

void launchFinish(DevWorld& w, int32_t n, float dt, bool clearForces)
{
	StepCounters* dc = devCounters(w);
	cudaMemsetAsync(&dc->bodyCount, 0, 2 * sizeof(uint32_t), w.stream);
	if (n > 0)
	{
		M3G_LAUNCH(kFinish, blocksFor(n, 256), 256, w.stream, w.B, n, dt, clearForces ? 1 : 0, dc);
	}
}

} // namespace m3g

// Narrowphase of one step: per contact, the armed tunnelling guard, the
// pose-delta manifold cache, regeneration with a speculative margin, anchor
// inheritance and separation offsets; then touch transitions turn into
// begin/end events and begin-touch wakes the sleeping partner.
// (reference src/world.cpp:1738-1845)
#include "m3d_dev.cuh"
#include "m3d_solve.cuh"

namespace m3g
{

// genRecord (null unless a differentiation tape records): per contact,
// kPrepRegenerated when the manifold was regenerated, kPrepHeld when the
// tunnelling guard held it, 0 when it was kept
__global__ void kNarrowphase(BodySoA B, ContactSoA C, int32_t maxCount, const uint32_t* countDev, float dt,
							 int8_t* transition, uint8_t* genRecord)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= maxCount)
	{
		return;
	}
	transition[c] = 0;
	if (genRecord != nullptr)
	{
		genRecord[c] = 0;
	}
	if (c >= (int)*countDev)
	{
		return;
	}
	int2 ab = C.bodies[c];
	if (!(B.bFlags[ab.x] & kBFAwake) && !(B.bFlags[ab.y] & kBFAwake))
	{
		return; // sleeping pair: nothing changes
	}
	uint8_t fl = C.flags[c];
	Xf xa = bodyXf(B, ab.x), xb = bodyXf(B, ab.y);
	if (fl & kCFTunnelGuard)
	{
		Manifold held;
		loadManifold(C, c, held);
		if (trackedMinSep(xa, xb, held) < -kLinearSlop)
		{
			if (genRecord != nullptr)
			{
				genRecord[c] = (uint8_t)kPrepHeld;
			}
			return; // keep the pre-crossing manifold, touching unchanged
		}
		fl &= (uint8_t)~kCFTunnelGuard;
	}
	int pc;
	if (!(fl & kCFHasCache) || poseChanged(xa, ld3(C.cachePosA[c]), ldq(C.cacheRotA[c])) ||
		poseChanged(xb, ld3(C.cachePosB[c]), ldq(C.cacheRotB[c])))
	{
		Manifold old, m;
		loadManifold(C, c, old);
		m = old;
		float relSpeed = len(sub(ld3(B.vel[ab.x]), ld3(B.vel[ab.y])));
		float margin = kSpeculativeBase + dt * relSpeed;
		const BodyCold& ca = B.cold[ab.x];
		const BodyCold& cb = B.cold[ab.y];
		collideShapes(ca.shape, xa, cb.shape, xb, margin, &m);
		inheritAnchors(old, m, ca.shape.type == kBox && cb.shape.type == kBox, xa, xb);
		fl |= kCFHasCache;
		C.cachePosA[c] = st3(xa.p);
		C.cacheRotA[c] = stq(xa.q);
		C.cachePosB[c] = st3(xb.p);
		C.cacheRotB[c] = stq(xb.q);
		setSeparationOffsets(m, xa, xb);
		storeManifold(C, c, m);
		pc = m.pointCount;
		if (genRecord != nullptr)
		{
			genRecord[c] = (uint8_t)kPrepRegenerated;
		}
	}
	else
	{
		pc = C.pointCount[c];
	}
	bool was = (fl & kCFTouching) != 0;
	bool now = pc > 0;
	fl = now ? (uint8_t)(fl | kCFTouching) : (uint8_t)(fl & ~kCFTouching);
	C.flags[c] = fl;
	transition[c] = (int8_t)(now && !was ? 1 : (!now && was ? -1 : 0));
}

__global__ void kTransitionFlags(const int8_t* transition, int32_t count, uint32_t* beginFlag, uint32_t* endFlag)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c < count)
	{
		int8_t t = transition[c];
		beginFlag[c] = t > 0 ? 1u : 0u;
		endFlag[c] = t < 0 ? 1u : 0u;
	}
}

__global__ void kTransitionEvents(const ContactSoA C, int32_t count, const int8_t* transition, const uint32_t* beginScan,
								  const uint32_t* endScan, int4* beginEv, int4* endEv)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= count)
	{
		return;
	}
	int8_t t = transition[c];
	if (t == 0)
	{
		return;
	}
	int2 ab = C.bodies[c];
	int4 ev = make_int4(ab.x, ab.y, (C.flags[c] & kCFSensor) ? 1 : 0, 0);
	if (t > 0)
	{
		beginEv[beginScan[c]] = ev;
	}
	else
	{
		endEv[endScan[c]] = ev;
	}
}

// Begin-touch wakes the sleeping partner of an awake body.  Every contact
// with a transition had an awake body when the narrowphase ran, so deciding
// from the awake bits of that moment gives the same set of wakes as the
// reference's serial loop (src/world.cpp:1817-1840).
__global__ void kWakeDecide(const BodySoA B, const ContactSoA C, int32_t count, const int8_t* transition,
							int32_t* target)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= count)
	{
		return;
	}
	int32_t t = -1;
	if (transition[c] > 0 && !(C.flags[c] & kCFSensor))
	{
		int2 ab = C.bodies[c];
		bool aw = (B.state[ab.x] & kStAwake) != 0, bw = (B.state[ab.y] & kStAwake) != 0;
		if (aw && !bw)
		{
			t = ab.y;
		}
		else if (bw && !aw)
		{
			t = ab.x;
		}
	}
	target[c] = t;
}

__global__ void kWakeApply(BodySoA B, int32_t count, const int32_t* target, uint32_t* stableDirty)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c < count && target[c] >= 0)
	{
		wakeBody(B, target[c], stableDirty);
	}
}

void launchNarrowphase(DevWorld& w, float dt)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	int32_t M = w.contactMax; // upper bound of the device contact count
	size_t c4 = (size_t)(M + 1) * sizeof(uint32_t);
	w.transition.ensure((size_t)M + 1);
	w.evBeginFlag.ensure(c4);
	w.evEndFlag.ensure(c4);
	w.removeScan.ensure(c4);
	w.moveSrc.ensure(c4);
	w.evBegin.ensure((size_t)(M + 1) * sizeof(int4));
	w.evEnd.ensure((size_t)(M + 1) * sizeof(int4));
	if (M <= 0)
	{
		fillWords(&dc->beginNP, 0u, 2 * sizeof(uint32_t), s);
		return;
	}
	int8_t* tr = w.transition.as<int8_t>();
	uint8_t* gen = nullptr;
	if (w.recording)
	{
		w.tapeGen.ensure((size_t)M + 1);
		gen = w.tapeGen.as<uint8_t>();
	}
	M3G_LAUNCH(kNarrowphase, blocksFor(M, 128), 128, s, w.B, w.C, M, &dc->contactCount, dt, tr, gen);
	M3G_LAUNCH(kTransitionFlags, blocksFor(M, 256), 256, s, tr, M, w.evBeginFlag.as<uint32_t>(),
			   w.evEndFlag.as<uint32_t>());
	uint32_t* beginScan = w.removeScan.as<uint32_t>();
	uint32_t* endScan = (uint32_t*)w.moveSrc.ptr;
	scanExclusive2(w.evBeginFlag.as<uint32_t>(), beginScan, M, &dc->beginNP, w.evEndFlag.as<uint32_t>(), endScan, M,
				   &dc->endNP, w.prim, s);
	M3G_LAUNCH(kTransitionEvents, blocksFor(M, 256), 256, s, w.C, M, tr, beginScan, endScan, w.evBegin.as<int4>(),
			   w.evEnd.as<int4>());
	int32_t* target = (int32_t*)w.evBeginFlag.ptr; // flags no longer needed
	M3G_LAUNCH(kWakeDecide, blocksFor(M, 256), 256, s, w.B, w.C, M, tr, target);
	M3G_LAUNCH(kWakeApply, blocksFor(M, 256), 256, s, w.B, M, target, stableDirtyWords(w));
}

} // namespace m3g

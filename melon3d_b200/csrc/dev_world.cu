// Device arena management: growth of the body and contact SoA arenas, the
// step counters, and the application of host-side API changes (body
// creation, setters, wake-ups) at the start of a step.
#include "m3d_dev.cuh"

#include <string.h>

namespace m3g
{

template <typename T>
static bool growArray(T*& p, int64_t oldCount, int64_t newCount, cudaStream_t s)
{
	T* np = nullptr;
	countAllocation();
	if (cudaMalloc((void**)&np, sizeof(T) * (size_t)newCount) != cudaSuccess)
	{
		return false;
	}
	cudaMemsetAsync(np, 0, sizeof(T) * (size_t)newCount, s);
	if (p != nullptr && oldCount > 0)
	{
		cudaMemcpyAsync(np, p, sizeof(T) * (size_t)oldCount, cudaMemcpyDeviceToDevice, s);
	}
	if (p != nullptr)
	{
		cudaStreamSynchronize(s);
		cudaFree(p);
	}
	p = np;
	return true;
}

bool growBodies(DevWorld& w, int32_t capacity)
{
	if (capacity <= w.bodyCap)
	{
		return true;
	}
	int32_t nc = w.bodyCap * 2 > capacity ? w.bodyCap * 2 : capacity;
	if (nc < 1024)
	{
		nc = 1024;
	}
	BodySoA& B = w.B;
	int64_t o = w.bodyCap;
	cudaStream_t s = w.stream;
	bool ok = true;
	ok &= growArray(B.pos, o, nc, s);
	ok &= growArray(B.rot, o, nc, s);
	ok &= growArray(B.vel, o, nc, s);
	ok &= growArray(B.angVel, o, nc, s);
	ok &= growArray(B.prevPos, o, nc, s);
	ok &= growArray(B.prevRot, o, nc, s);
	ok &= growArray(B.prevVel, o, nc, s);
	ok &= growArray(B.prevAngVel, o, nc, s);
	ok &= growArray(B.massInv, o, nc, s);
	ok &= growArray(B.iw0, o, nc, s);
	ok &= growArray(B.iw1, o, nc, s);
	ok &= growArray(B.iw2, o, nc, s);
	ok &= growArray(B.force, o, nc, s);
	ok &= growArray(B.torque, o, nc, s);
	ok &= growArray(B.sleep, o, nc, s);
	ok &= growArray(B.state, o, nc, s);
	ok &= growArray(B.cold, o, nc, s);
	ok &= growArray(B.fatLo, o, nc, s);
	ok &= growArray(B.fatHi, o, nc, s);
	ok &= growArray(B.hasFat, o, nc, s);
	ok &= growArray(B.moved, o, nc, s);
	ok &= growArray(B.isActive, o, nc, s);
	ok &= growArray(B.isStable, o, nc, s);
	ok &= growArray(B.inStableTier, o, nc, s);
	ok &= growArray(B.inStableCells, o, nc, s);
	ok &= growArray(B.bFlags, o, nc, s);
	B.capacity = nc;
	w.bodyCap = nc;
	return ok;
}

// point arrays are slot-major: each slot block moves to its new offset
template <typename T>
static bool growPointArray(T*& p, int64_t oldCap, int64_t newCap, cudaStream_t s)
{
	T* np = nullptr;
	countAllocation();
	if (cudaMalloc((void**)&np, sizeof(T) * (size_t)newCap * 4) != cudaSuccess)
	{
		return false;
	}
	cudaMemsetAsync(np, 0, sizeof(T) * (size_t)newCap * 4, s);
	if (p != nullptr)
	{
		for (int slot = 0; slot < 4; ++slot)
		{
			cudaMemcpyAsync(np + slot * newCap, p + slot * oldCap, sizeof(T) * (size_t)oldCap,
							cudaMemcpyDeviceToDevice, s);
		}
		cudaStreamSynchronize(s);
		cudaFree(p);
	}
	p = np;
	return true;
}

bool growContacts(DevWorld& w, int32_t capacity)
{
	if (capacity <= w.contactCap)
	{
		return true;
	}
	int32_t nc = w.contactCap * 2 > capacity ? w.contactCap * 2 : capacity;
	if (nc < 4096)
	{
		nc = 4096;
	}
	ContactSoA& C = w.C;
	int64_t o = w.contactCap;
	cudaStream_t s = w.stream;
	bool ok = true;
	ok &= growArray(C.bodies, o, nc, s);
	ok &= growArray(C.pointCount, o, nc, s);
	ok &= growArray(C.flags, o, nc, s);
	ok &= growArray(C.normal, o, nc, s);
	ok &= growArray(C.mat, o, nc, s);
	ok &= growArray(C.cachePosA, o, nc, s);
	ok &= growArray(C.cacheRotA, o, nc, s);
	ok &= growArray(C.cachePosB, o, nc, s);
	ok &= growArray(C.cacheRotB, o, nc, s);
	ok &= growPointArray(C.pAnchorA, o, nc, s);
	ok &= growPointArray(C.pAnchorB, o, nc, s);
	ok &= growPointArray(C.pFricA, o, nc, s);
	ok &= growPointArray(C.pFricB, o, nc, s);
	ok &= growPointArray(C.pSlip, o, nc, s);
	ok &= growPointArray(C.pRA, o, nc, s);
	ok &= growPointArray(C.pRB, o, nc, s);
	ok &= growPointArray(C.pJA, o, nc, s);
	ok &= growPointArray(C.pJB, o, nc, s);
	C.capacity = nc;
	w.contactCap = nc;
	if (w.batched)
	{
		// the re-layout target: same capacity, no contents to keep
		ContactSoA& D = w.C2;
		ok &= growArray(D.bodies, 0, nc, s);
		ok &= growArray(D.pointCount, 0, nc, s);
		ok &= growArray(D.flags, 0, nc, s);
		ok &= growArray(D.normal, 0, nc, s);
		ok &= growArray(D.mat, 0, nc, s);
		ok &= growArray(D.cachePosA, 0, nc, s);
		ok &= growArray(D.cacheRotA, 0, nc, s);
		ok &= growArray(D.cachePosB, 0, nc, s);
		ok &= growArray(D.cacheRotB, 0, nc, s);
		ok &= growPointArray(D.pAnchorA, 0, nc, s);
		ok &= growPointArray(D.pAnchorB, 0, nc, s);
		ok &= growPointArray(D.pFricA, 0, nc, s);
		ok &= growPointArray(D.pFricB, 0, nc, s);
		ok &= growPointArray(D.pSlip, 0, nc, s);
		ok &= growPointArray(D.pRA, 0, nc, s);
		ok &= growPointArray(D.pRB, 0, nc, s);
		ok &= growPointArray(D.pJA, 0, nc, s);
		ok &= growPointArray(D.pJB, 0, nc, s);
		D.capacity = nc;
	}
	return ok;
}

StepCounters* devCounters(DevWorld& w)
{
	if (w.counters.ptr == nullptr)
	{
		w.counters.ensure(sizeof(StepCounters));
		cudaMemsetAsync(w.counters.ptr, 0, sizeof(StepCounters), w.stream);
		cudaMallocHost((void**)&w.hostCounters, sizeof(StepCounters));
		memset(w.hostCounters, 0, sizeof(StepCounters));
		w.prim.errorWord = &w.counters.as<StepCounters>()->waitErrors;
	}
	return w.counters.as<StepCounters>();
}

uint32_t* stableDirtyWords(DevWorld& w)
{
	if (w.batched)
	{
		return w.worldStableDirty.as<uint32_t>();
	}
	return &devCounters(w)->stableDirty;
}

__global__ void kSetU32(uint32_t* p, uint32_t v) { M3G_KERNEL_BEGIN(); *p = v; }

void setDeviceCount(DevWorld& w, uint32_t* p, uint32_t v) { M3G_LAUNCH(kSetU32, 1, 1, w.stream, p, v); }

__global__ void kResetCounters(StepCounters* c, uint32_t contactCount)
{
	M3G_KERNEL_BEGIN();
	uint32_t* words = (uint32_t*)c;
	for (int i = threadIdx.x; i < (int)(sizeof(StepCounters) / sizeof(uint32_t)); i += blockDim.x)
	{
		words[i] = 0u;
	}
	__syncthreads();
	if (threadIdx.x == 0)
	{
		c->contactCount = contactCount;
	}
}

void resetStepCounters(DevWorld& w, uint32_t contactCount)
{
	M3G_LAUNCH(kResetCounters, 1, 128, w.stream, devCounters(w), contactCount);
}

void readCounters(DevWorld& w)
{
	devCounters(w);
	cudaMemcpyAsync(w.hostCounters, w.counters.ptr, sizeof(StepCounters), cudaMemcpyDeviceToHost, w.stream);
	cudaStreamSynchronize(w.stream);
}

// ---- uploads ----------------------------------------------------------------

__global__ void kApplyUploads(BodySoA B, const BodyUpload* recs, int32_t count, uint8_t* matDirty)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= count)
	{
		return;
	}
	const BodyUpload& u = recs[k];
	int i = u.index;
	uint32_t m = u.mask;
	if (m & kUpAll)
	{
		float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		B.prevPos[i] = z;
		B.prevRot[i] = z;
		B.prevVel[i] = z;
		B.prevAngVel[i] = z;
		B.massInv[i] = u.massInv;
		B.cold[i] = u.cold;
		m |= kUpPose | kUpVel | kUpIW | kUpForce | kUpState | kUpFatReset;
	}
	if (m & kUpPose)
	{
		B.pos[i] = u.pos;
		B.rot[i] = u.rot;
	}
	if (m & kUpVel)
	{
		B.vel[i] = u.vel;
		B.angVel[i] = u.angVel;
	}
	if (m & kUpIW)
	{
		B.iw0[i] = u.iw0;
		B.iw1[i] = u.iw1;
		B.iw2[i] = u.iw2;
	}
	if (m & kUpForce)
	{
		B.force[i] = u.force;
		B.torque[i] = u.torque;
	}
	if (m & kUpState)
	{
		B.state[i] = (uint8_t)u.state;
		B.sleep[i] = u.sleep;
	}
	if (m & kUpCold)
	{
		B.cold[i] = u.cold;
		matDirty[i] = 1;
	}
	if (m & kUpFatReset)
	{
		B.hasFat[i] = 0;
	}
}

void launchApplyUploads(DevWorld& w, const BodyUpload* hostRecs, int32_t count)
{
	if (count <= 0)
	{
		return;
	}
	w.uploads.ensure(sizeof(BodyUpload) * (size_t)count);
	w.matDirty.ensureZeroed((size_t)w.bodyCap, w.stream);
	cudaMemcpyAsync(w.uploads.ptr, hostRecs, sizeof(BodyUpload) * (size_t)count, cudaMemcpyHostToDevice, w.stream);
	M3G_LAUNCH(kApplyUploads, blocksFor(count, 128), 128, w.stream, w.B, w.uploads.as<BodyUpload>(), count,
																w.matDirty.as<uint8_t>());
}

// combined materials of every live contact of a body whose material changed
// (reference src/world.cpp:804-818)
__global__ void kMaterialRefresh(BodySoA B, ContactSoA C, int32_t count, uint8_t* matDirty)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= count)
	{
		return;
	}
	int2 ab = C.bodies[c];
	if (!matDirty[ab.x] && !matDirty[ab.y])
	{
		return;
	}
	const BodyCold& a = B.cold[ab.x];
	const BodyCold& b = B.cold[ab.y];
	float4 nf = C.normal[c];
	nf.w = sqrtf(a.friction * b.friction);
	C.normal[c] = nf;
	C.mat[c] = make_float2(a.restitution > b.restitution ? a.restitution : b.restitution,
						   sqrtf(a.rollingResistance * b.rollingResistance));
}

void launchMaterialRefresh(DevWorld& w)
{
	w.matDirty.ensureZeroed((size_t)w.bodyCap, w.stream);
	if (w.contactCount > 0)
	{
		M3G_LAUNCH(kMaterialRefresh, blocksFor(w.contactCount, 256), 256, w.stream, w.B, w.C, w.contactCount,
																				 w.matDirty.as<uint8_t>());
	}
	cudaMemsetAsync(w.matDirty.ptr, 0, (size_t)w.bodyCap, w.stream);
}

} // namespace m3g

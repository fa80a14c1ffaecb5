// Host side of the GPU world: the C API of include/melon3d.h.
//
// The world's state lives in HBM (DevWorld).  The host keeps
//  - the slot allocator (free lists + generations), joint table and the
//    per-body records the API reads and writes (a mirror of the device
//    state, refreshed lazily by one bulk copy after a step);
//  - the list of bodies changed through the API since the last step, which
//    is uploaded at the start of the next step;
//  - the contacts' (bodyA, bodyB, flags) sidecar, downloaded only when a body
//    is destroyed, so destroy-time contact removal and end events follow the
//    reference exactly.
// m3d_world_step drives the device stages in the reference's order
// (src/world.cpp:1437-2167) and returns once the step's events and counters
// are on the host.
#include "m3d_collide.cuh"
#include "m3d_dev.cuh"
#include "melon3d.h"
#include "melon3d_debug.h"
#include "melon3d_gpu.h"

#include <chrono>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

using namespace m3g;

namespace
{

using Clock = std::chrono::steady_clock;

float toMs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<float, std::milli>(b - a).count(); }

struct HostBody
{
	m3d_vec3 position;
	m3d_quat rotation;
	m3d_vec3 linearVelocity;
	m3d_vec3 angularVelocity;
	float invMass;
	m3d_vec3 invInertiaLocal;
	m3d_mat3 invInertiaWorld;
	float mass;
	m3d_vec3 force;
	m3d_vec3 torque;
	float sleepTime;
	float smoothedEnergy;
	bool enableSleep;
	bool isAwake;
	bool inUse;
	bool isSensor;
	uint32_t generation;
	uint64_t userData;
	BodyCold cold;
};

} // namespace

struct m3d_world
{
	m3d_world_def def;
	DevWorld dev;

	std::vector<HostBody> bodies;
	std::vector<int32_t> freeBodies;
	std::vector<JointRec> joints;
	std::vector<int32_t> freeJoints;
	bool jointsDirty = true;
	std::vector<uint64_t> jointedPairs;
	bool jointedPairsDirty = true;

	std::vector<uint32_t> dirtyMask;
	std::vector<int32_t> dirtyList;
	bool anyMaterialChange = false;

	bool gridDirty = true;
	bool stableDirty = true;
	bool stableForce = false;
	int32_t stepsSinceStableBuild = 1000;
	bool anyForcesApplied = false;
	bool mirrorStale = false; // device bodies newer than the host records
	bool awakeStale = false;  // device awake bits newer than the host records
	// the device's awake bits as a destroy downloaded them (while awakeStale,
	// until the device or the host records change); read per body on demand
	std::vector<uint8_t> awakeBits;
	bool awakeBitsValid = false;

	// contact sidecar (valid between a step and the next flush): the device's
	// contact bodies and flags and its per-body contact lists (CSR over the
	// original contact indices), downloaded into pinned memory by the first
	// destroy after a step
	bool contactMirrorValid = false;
	int2* cBodies = nullptr;      // cCount live slots
	uint8_t* cFlags = nullptr;
	uint32_t* adjStart = nullptr; // adjBodies + 1 offsets into adjList
	int32_t* adjList = nullptr;
	int32_t cCount = 0;
	int32_t adjBodies = 0;
	int64_t sideContactCap = 0, sideBodyCap = 0;
	// cPerm: original device index of each slot; cPos: current slot of each
	// original contact (-1: removed).  Both are the identity outside the
	// indices listed in cTouched, which the flush restores.
	std::vector<int32_t> cPerm;
	std::vector<int32_t> cPos;
	std::vector<int32_t> cTouched;
	bool contactsEdited = false;

	std::vector<m3d_contact_event> beginEvents;
	std::vector<m3d_contact_event> endEvents;
	m3d_profile profile;

	cudaEvent_t evStart = nullptr, evStop = nullptr;
	float lastDeviceMs = 0.0f;
	int32_t status = M3D_GPU_OK;
	char errorText[256] = { 0 };

	// a batch of worlds packed into this one (m3d_gpu_batch_create): per world,
	// its first body slot and its own stable-tier schedule; empty otherwise
	std::vector<int32_t> batchFirstBody; // worlds + 1 entries
	std::vector<uint32_t> bodyWorld;     // world of each body slot
	std::vector<uint8_t> batchStableDirty, batchStableForce, batchRebuild;
	std::vector<int32_t> batchStepsSinceStableBuild;
	bool stepped = false;
	// the last step was a no-op that ended with every body asleep (see
	// m3d_world_step); any API edit clears it
	bool quiescent = false;
	int64_t quiescentSteps = 0; // steps taken by the sleeping-world fast path
	bool lastRebuiltStable = false; // the last step rebuilt the stable tier
	// online autotuning of the serial-island kernel choice (m3d_gpu_autotune)
	struct Tune
	{
		std::vector<int2> candidates; // (tinyContacts, tinyModeIslands)
		std::vector<std::vector<float>> samples;
		int32_t stepsPerTrial = 0, rounds = 0, step = 0;
		bool active = false, done = false;
		int32_t chosen = -1;
		std::string key;
	} tune;

	// differentiation tape (m3d_gpu_tape_begin); null when not recording
	DiffTape* tape = nullptr;

	// pinned staging
	std::vector<BodyUpload> uploadRecs;
	float4* pinPos = nullptr;
	float4* pinRot = nullptr;
	float4* pinVel = nullptr;
	float4* pinAng = nullptr;
	uint8_t* pinState = nullptr;
	float2* pinSleep = nullptr;
	int32_t pinCap = 0;
	// the step's three event lists (removal ends, begins, ends), pinCap each,
	// and a batch's per-world stable-dirty words
	int4* pinEvents = nullptr;
	int32_t pinEventCap = 0;
	uint32_t* pinWorldDirty = nullptr;
	int32_t pinWorldDirtyCap = 0;
	// the destroy download issued right after a step that followed destroys
	// (on its own stream, so it overlaps the host's work until the next
	// destroy); sideN bodies, sideC contacts, the awake bits in pinSideState
	cudaStream_t sideStream = nullptr;
	cudaEvent_t sideDone = nullptr;
	PrimScratch sidePrim;
	uint8_t* pinSideState = nullptr;
	int32_t pinSideCap = 0;
	bool sidecarPending = false;
	int32_t sideN = 0, sideC = 0;
	int32_t destroysSinceStep = 0;
};

namespace
{

void setError(m3d_world* w, int32_t code, const char* what)
{
	if (w->status == M3D_GPU_OK)
	{
		w->status = code;
		snprintf(w->errorText, sizeof(w->errorText), "%s", what);
		fprintf(stderr, "melon3d_gpu: %s\n", what);
	}
}

void checkCuda(m3d_world* w, const char* where)
{
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess)
	{
		char buf[256];
		snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
		setError(w, M3D_GPU_ERR_CUDA, buf);
	}
}

HostBody* getBody(m3d_world* w, m3d_body_id id)
{
	if (id.index < 0 || id.index >= (int32_t)w->bodies.size())
	{
		return nullptr;
	}
	HostBody& b = w->bodies[id.index];
	if (!b.inUse || b.generation != id.generation)
	{
		return nullptr;
	}
	return &b;
}

m3d_body_id makeId(m3d_world* w, int32_t index) { return { index, w->bodies[index].generation }; }

void markDirty(m3d_world* w, int32_t index, uint32_t mask)
{
	w->quiescent = false;
	if ((int32_t)w->dirtyMask.size() < (int32_t)w->bodies.size())
	{
		w->dirtyMask.resize(w->bodies.size(), 0);
	}
	if (w->dirtyMask[index] == 0)
	{
		w->dirtyList.push_back(index);
	}
	w->dirtyMask[index] |= mask;
}

bool isBatch(const m3d_world* w) { return !w->batchFirstBody.empty(); }

// the stable tier of the body's world is out of date (and, with force, is
// rebuilt at the next step whatever its schedule)
void markStableDirty(m3d_world* w, int32_t index, bool force = false)
{
	w->quiescent = false;
	if (isBatch(w))
	{
		const uint32_t k = w->bodyWorld[index];
		w->batchStableDirty[k] = 1;
		if (force)
		{
			w->batchStableForce[k] = 1;
		}
		return;
	}
	w->stableDirty = true;
	if (force)
	{
		w->stableForce = true;
	}
}

uint32_t stateBits(const HostBody& b)
{
	return (b.inUse ? kStInUse : 0) | (b.isAwake ? kStAwake : 0) | (b.enableSleep ? kStEnableSleep : 0) |
		   (b.isSensor ? kStSensor : 0);
}

void ensurePinned(m3d_world* w, int32_t n)
{
	if (n <= w->pinCap)
	{
		return;
	}
	int32_t cap = w->pinCap * 2 > n ? w->pinCap * 2 : n;
	cap = cap < 1024 ? 1024 : cap;
	cudaFreeHost(w->pinPos);
	cudaFreeHost(w->pinRot);
	cudaFreeHost(w->pinVel);
	cudaFreeHost(w->pinAng);
	cudaFreeHost(w->pinState);
	cudaFreeHost(w->pinSleep);
	cudaMallocHost((void**)&w->pinPos, sizeof(float4) * cap);
	cudaMallocHost((void**)&w->pinRot, sizeof(float4) * cap);
	cudaMallocHost((void**)&w->pinVel, sizeof(float4) * cap);
	cudaMallocHost((void**)&w->pinAng, sizeof(float4) * cap);
	cudaMallocHost((void**)&w->pinState, sizeof(uint8_t) * cap);
	cudaMallocHost((void**)&w->pinSleep, sizeof(float2) * cap);
	w->pinCap = cap;
}

// Refresh the host mirror from the device after a step (one bulk copy).
void syncMirror(m3d_world* w)
{
	if (!w->mirrorStale)
	{
		return;
	}
	int32_t n = (int32_t)w->bodies.size();
	if (n > 0)
	{
		ensurePinned(w, n);
		DevWorld& d = w->dev;
		cudaStream_t s = d.stream;
		cudaMemcpyAsync(w->pinPos, d.B.pos, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(w->pinRot, d.B.rot, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(w->pinVel, d.B.vel, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(w->pinAng, d.B.angVel, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(w->pinState, d.B.state, sizeof(uint8_t) * n, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(w->pinSleep, d.B.sleep, sizeof(float2) * n, cudaMemcpyDeviceToHost, s);
		cudaStreamSynchronize(s);
		checkCuda(w, "mirror download");
		bool anyDirty = !w->dirtyList.empty();
		for (int32_t i = 0; i < n; ++i)
		{
			HostBody& b = w->bodies[i];
			// fields changed through the API since the step are newer on the
			// host; a body created since the step has no device state yet
			uint32_t dm = (anyDirty && i < (int32_t)w->dirtyMask.size()) ? w->dirtyMask[i] : 0u;
			if (!b.inUse || (dm & kUpAll))
			{
				continue;
			}
			if (!(dm & kUpPose))
			{
				b.position = m3d_v3(w->pinPos[i].x, w->pinPos[i].y, w->pinPos[i].z);
				b.rotation = { w->pinRot[i].x, w->pinRot[i].y, w->pinRot[i].z, w->pinRot[i].w };
			}
			if (!(dm & kUpVel))
			{
				b.linearVelocity = m3d_v3(w->pinVel[i].x, w->pinVel[i].y, w->pinVel[i].z);
				b.angularVelocity = m3d_v3(w->pinAng[i].x, w->pinAng[i].y, w->pinAng[i].z);
			}
			if (!(dm & kUpState))
			{
				b.isAwake = (w->pinState[i] & kStAwake) != 0;
				b.sleepTime = w->pinSleep[i].x;
				b.smoothedEnergy = w->pinSleep[i].y;
			}
		}
	}
	w->mirrorStale = false;
	w->awakeStale = false;
	w->awakeBitsValid = false;
}

// RemoveContactAt on the host sidecar (reference src/world.cpp:100-119)
void removeContactAt(m3d_world* w, int32_t i)
{
	int32_t last = w->cCount - 1;
	int32_t gone = w->cPerm[i];
	w->cPos[gone] = -1;
	w->cTouched.push_back(gone);
	w->cTouched.push_back(i);
	if (i != last)
	{
		w->cBodies[i] = w->cBodies[last];
		w->cFlags[i] = w->cFlags[last];
		w->cPerm[i] = w->cPerm[last];
		w->cPos[w->cPerm[i]] = i;
		w->cTouched.push_back(w->cPerm[i]);
	}
	--w->cCount;
	w->contactsEdited = true;
}

void ensureSidecar(m3d_world* w, int32_t n, int32_t c)
{
	if (c > w->sideContactCap)
	{
		int64_t cap = w->sideContactCap * 2 > c ? w->sideContactCap * 2 : c;
		cap = cap < 4096 ? 4096 : cap;
		cudaFreeHost(w->cBodies);
		cudaFreeHost(w->cFlags);
		cudaFreeHost(w->adjList);
		cudaMallocHost((void**)&w->cBodies, sizeof(int2) * cap);
		cudaMallocHost((void**)&w->cFlags, sizeof(uint8_t) * cap);
		cudaMallocHost((void**)&w->adjList, sizeof(int32_t) * 2 * cap);
		w->sideContactCap = cap;
	}
	if (n + 1 > w->sideBodyCap)
	{
		int64_t cap = w->sideBodyCap * 2 > n + 1 ? w->sideBodyCap * 2 : n + 1;
		cap = cap < 4096 ? 4096 : cap;
		cudaFreeHost(w->adjStart);
		cudaMallocHost((void**)&w->adjStart, sizeof(uint32_t) * cap);
		w->sideBodyCap = cap;
	}
}

// Everything a destroy reads from the device, in one download and one wait:
// the awake bits when the device's are newer than the host records, and once
// per step the contact sidecar, whose per-body contact lists are built on the
// device.
// Issue on stream s what a destroy reads from the device: the awake bits of n
// bodies into `state`, and the contact sidecar of c contacts, whose per-body
// contact lists are built on the device (scan scratch prim).
void enqueueDestroyDownload(m3d_world* w, cudaStream_t s, PrimScratch& prim, bool awake, bool contacts, int32_t n,
							int32_t c, uint8_t* state)
{
	DevWorld& d = w->dev;
	if (awake && n > 0)
	{
		cudaMemcpyAsync(state, d.B.state, sizeof(uint8_t) * n, cudaMemcpyDeviceToHost, s);
	}
	if (contacts && c > 0)
	{
		ensureSidecar(w, n, c);
		launchContactAdjacency(d, n, s, prim);
		cudaMemcpyAsync(w->cBodies, d.C.bodies, sizeof(int2) * c, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(w->cFlags, d.C.flags, sizeof(uint8_t) * c, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(w->adjStart, d.adjStart.ptr, sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(w->adjList, d.adjList.ptr, sizeof(int32_t) * 2 * c, cudaMemcpyDeviceToHost, s);
	}
}

// Take a completed destroy download: the awake bits of the first n bodies
// (kept aside and read per body by hostAwake), the contact sidecar of c
// contacts.
void applyDestroyDownload(m3d_world* w, bool awake, bool contacts, int32_t n, int32_t c, const uint8_t* state)
{
	if (awake)
	{
		w->awakeBits.assign(state, state + (n > 0 ? n : 0));
		w->awakeBitsValid = true;
	}
	if (contacts)
	{
		w->cCount = c;
		w->adjBodies = c > 0 ? n : 0;
		int32_t had = (int32_t)w->cPerm.size();
		if (had < c)
		{
			w->cPerm.resize(c);
			w->cPos.resize(c);
			for (int32_t i = had; i < c; ++i)
			{
				w->cPerm[i] = i;
				w->cPos[i] = i;
			}
		}
		w->contactMirrorValid = true;
		w->contactsEdited = false;
	}
}

// A streaming world destroys after most steps: right after a step that
// followed destroys, the download the next destroy needs is issued on a
// second stream and left running.  Nothing on the device changes until the
// next step or flush, both of which first drop it (dropSidecar).
void prefetchSidecar(m3d_world* w)
{
	DevWorld& d = w->dev;
	if (w->sideStream == nullptr)
	{
		cudaStreamCreateWithFlags(&w->sideStream, cudaStreamNonBlocking);
		cudaEventCreateWithFlags(&w->sideDone, cudaEventDisableTiming);
		w->sidePrim.errorWord = d.prim.errorWord;
	}
	w->sidePrim.waitLimit = d.prim.waitLimit;
	const int32_t n = (int32_t)w->bodies.size();
	const int32_t c = d.contactCount;
	if (n > w->pinSideCap)
	{
		cudaFreeHost(w->pinSideState);
		int32_t cap = n * 2 > 1024 ? n * 2 : 1024;
		cudaMallocHost((void**)&w->pinSideState, cap);
		w->pinSideCap = cap;
	}
	enqueueDestroyDownload(w, w->sideStream, w->sidePrim, true, true, n, c, w->pinSideState);
	cudaEventRecord(w->sideDone, w->sideStream);
	w->sidecarPending = true;
	w->sideN = n;
	w->sideC = c;
}

// Forget a prefetched destroy download (the device is about to change), once
// its copies have landed.
void dropSidecar(m3d_world* w)
{
	if (w->sidecarPending)
	{
		cudaEventSynchronize(w->sideDone);
		w->sidecarPending = false;
	}
}

// Everything a destroy reads from the device, in one download and one wait:
// the awake bits when the device's are newer than the host records, and once
// per step the contact sidecar, whose per-body contact lists are built on the
// device.  Taken from the prefetch when one is pending.
void prepareDestroy(m3d_world* w)
{
	const bool awake = w->awakeStale && !w->awakeBitsValid;
	const bool contacts = !w->contactMirrorValid;
	if (!awake && !contacts)
	{
		return;
	}
	if (w->sidecarPending && contacts)
	{
		cudaEventSynchronize(w->sideDone);
		w->sidecarPending = false;
		checkCuda(w, "destroy download");
		applyDestroyDownload(w, awake, contacts, w->sideN, w->sideC, w->pinSideState);
		return;
	}
	dropSidecar(w);
	DevWorld& d = w->dev;
	const int32_t n = (int32_t)w->bodies.size();
	const int32_t c = d.contactCount;
	if (awake && n > 0)
	{
		ensurePinned(w, n);
	}
	enqueueDestroyDownload(w, d.stream, d.prim, awake, contacts, n, c, w->pinState);
	cudaStreamSynchronize(d.stream);
	checkCuda(w, "destroy download");
	applyDestroyDownload(w, awake, contacts, n, c, w->pinState);
}

// Whether a body is awake: the host record when it is current (edited since
// the step, or refreshed from the device), else the bits a destroy downloaded.
bool hostAwake(m3d_world* w, int32_t i)
{
	if (w->awakeStale && w->awakeBitsValid && i < (int32_t)w->awakeBits.size())
	{
		uint32_t dm = i < (int32_t)w->dirtyMask.size() ? w->dirtyMask[i] : 0u;
		if (!(dm & (kUpAll | kUpState)))
		{
			return (w->awakeBits[i] & kStAwake) != 0;
		}
	}
	return w->bodies[i].isAwake;
}

void wakeBodyHost(m3d_world* w, int32_t index)
{
	HostBody& b = w->bodies[index];
	if (b.cold.type == kStatic)
	{
		return;
	}
	if (!hostAwake(w, index))
	{
		markStableDirty(w, index);
	}
	b.isAwake = true;
	b.sleepTime = 0.0f;
	b.smoothedEnergy = 4.0f * kSleepEnergyThresh;
	markDirty(w, index, kUpState);
}

m3d_mat3 toMat(const M3& m)
{
	m3d_mat3 r;
	r.cx = m3d_v3(m.cx.x, m.cx.y, m.cx.z);
	r.cy = m3d_v3(m.cy.x, m.cy.y, m.cy.z);
	r.cz = m3d_v3(m.cz.x, m.cz.y, m.cz.z);
	return r;
}

void updateInvInertiaWorld(HostBody& b)
{
	M3 m = invInertiaWorld(q4(b.rotation.x, b.rotation.y, b.rotation.z, b.rotation.w),
						   v3(b.invInertiaLocal.x, b.invInertiaLocal.y, b.invInertiaLocal.z));
	b.invInertiaWorld = toMat(m);
}

// mass, inverse mass and local inverse inertia (reference src/world.cpp:46-98)
void computeMassProperties(HostBody& body, const m3d_shape_def* def)
{
	float density = def->density > 0.0f ? def->density : 1000.0f;
	float mass = 0.0f;
	m3d_vec3 inertia = m3d_v3_zero();
	switch (def->type)
	{
		case M3D_SHAPE_SPHERE:
		{
			float r = def->radius;
			mass = density * (4.0f / 3.0f) * M3D_PI * r * r * r;
			float i = 0.4f * mass * r * r;
			inertia = m3d_v3(i, i, i);
			break;
		}
		case M3D_SHAPE_BOX:
		{
			m3d_vec3 e = def->halfExtents;
			mass = density * 8.0f * e.x * e.y * e.z;
			inertia = m3d_v3(mass / 3.0f * (e.y * e.y + e.z * e.z), mass / 3.0f * (e.x * e.x + e.z * e.z),
							 mass / 3.0f * (e.x * e.x + e.y * e.y));
			break;
		}
		case M3D_SHAPE_CAPSULE:
		{
			float r = def->radius;
			float h = def->halfHeight;
			float mc = density * M3D_PI * r * r * (2.0f * h);
			float ms = density * (4.0f / 3.0f) * M3D_PI * r * r * r;
			mass = mc + ms;
			float iy = 0.5f * mc * r * r + 0.4f * ms * r * r;
			float d = h + 0.375f * r;
			float ixz = mc * (0.25f * r * r + h * h / 3.0f) + (83.0f / 320.0f) * ms * r * r + ms * d * d;
			inertia = m3d_v3(ixz, iy, ixz);
			break;
		}
	}
	body.mass = mass;
	if (body.cold.type == kDynamic && mass > 0.0f)
	{
		body.invMass = 1.0f / mass;
		body.invInertiaLocal = m3d_v3(inertia.x > 0.0f ? 1.0f / inertia.x : 0.0f, inertia.y > 0.0f ? 1.0f / inertia.y : 0.0f,
									  inertia.z > 0.0f ? 1.0f / inertia.z : 0.0f);
	}
	else
	{
		body.invMass = 0.0f;
		body.invInertiaLocal = m3d_v3_zero();
	}
}

float4 f4(m3d_vec3 v) { return make_float4(v.x, v.y, v.z, 0.0f); }
float4 f4q(m3d_quat q) { return make_float4(q.x, q.y, q.z, q.w); }

// Upload every body touched through the API, apply destroy-time contact
// removals, refresh materials, joints and the jointed-pair list.
void flushHostChanges(m3d_world* w)
{
	DevWorld& d = w->dev;
	int32_t n = (int32_t)w->bodies.size();
	if (w->sidecarPending && (n + 1 > d.bodyCap || !w->dirtyList.empty() || (w->contactMirrorValid && w->contactsEdited) ||
							  w->anyMaterialChange || w->jointsDirty || w->jointedPairsDirty))
	{
		dropSidecar(w); // the device is about to change under the prefetch
	}
	if (!w->dirtyList.empty())
	{
		w->awakeBitsValid = false; // uploads change the device, edit masks are cleared
	}
	if (!growBodies(d, n + 1))
	{
		setError(w, M3D_GPU_ERR_ALLOC, "body arena growth failed");
	}
	if (!w->dirtyList.empty())
	{
		w->uploadRecs.resize(w->dirtyList.size());
		for (size_t k = 0; k < w->dirtyList.size(); ++k)
		{
			int32_t i = w->dirtyList[k];
			const HostBody& b = w->bodies[i];
			BodyUpload& u = w->uploadRecs[k];
			memset(&u, 0, sizeof(u));
			u.index = i;
			u.mask = w->dirtyMask[i];
			u.pos = f4(b.position);
			u.rot = f4q(b.rotation);
			u.vel = f4(b.linearVelocity);
			u.angVel = f4(b.angularVelocity);
			u.massInv = make_float4(b.invMass, b.invInertiaLocal.x, b.invInertiaLocal.y, b.invInertiaLocal.z);
			u.iw0 = f4(b.invInertiaWorld.cx);
			u.iw1 = f4(b.invInertiaWorld.cy);
			u.iw2 = f4(b.invInertiaWorld.cz);
			u.force = f4(b.force);
			u.torque = f4(b.torque);
			u.sleep = make_float2(b.sleepTime, b.smoothedEnergy);
			u.state = stateBits(b);
			u.cold = b.cold;
			w->dirtyMask[i] = 0;
		}
		launchApplyUploads(d, w->uploadRecs.data(), (int32_t)w->uploadRecs.size());
		w->dirtyList.clear();
	}
	if (w->contactMirrorValid && w->contactsEdited)
	{
		// destroy-time swap-removes: move the survivors the host moved (only
		// slots listed in cTouched can differ from the identity)
		std::sort(w->cTouched.begin(), w->cTouched.end());
		w->cTouched.erase(std::unique(w->cTouched.begin(), w->cTouched.end()), w->cTouched.end());
		std::vector<int2> moves;
		for (int32_t k : w->cTouched)
		{
			if (k < w->cCount && w->cPerm[k] != k)
			{
				moves.push_back(make_int2(k, w->cPerm[k]));
			}
		}
		launchContactMoves(d, moves.data(), (int32_t)moves.size());
		d.contactCount = w->cCount;
		w->contactsEdited = false;
	}
	for (int32_t k : w->cTouched)
	{
		w->cPerm[k] = k;
		w->cPos[k] = k;
	}
	w->cTouched.clear();
	w->contactMirrorValid = false;
	if (w->anyMaterialChange)
	{
		launchMaterialRefresh(d);
		w->anyMaterialChange = false;
	}
	if (w->jointsDirty)
	{
		d.jointCount = (int32_t)w->joints.size();
		if (d.jointCount > 0)
		{
			d.joints.ensure(sizeof(JointRec) * w->joints.size());
			cudaMemcpyAsync(d.joints.ptr, w->joints.data(), sizeof(JointRec) * w->joints.size(), cudaMemcpyHostToDevice,
							d.stream);
		}
		w->jointsDirty = false;
	}
	if (w->jointedPairsDirty)
	{
		w->jointedPairs.clear();
		for (const JointRec& j : w->joints)
		{
			if (j.inUse)
			{
				int32_t lo = j.bodyA < j.bodyB ? j.bodyA : j.bodyB;
				int32_t hi = j.bodyA < j.bodyB ? j.bodyB : j.bodyA;
				w->jointedPairs.push_back(((uint64_t)(uint32_t)lo << 32) | (uint32_t)hi);
			}
		}
		std::sort(w->jointedPairs.begin(), w->jointedPairs.end());
		d.jointedCount = (int32_t)w->jointedPairs.size();
		if (d.jointedCount > 0)
		{
			d.jointedPairs.ensure(sizeof(uint64_t) * w->jointedPairs.size());
			cudaMemcpyAsync(d.jointedPairs.ptr, w->jointedPairs.data(), sizeof(uint64_t) * w->jointedPairs.size(),
							cudaMemcpyHostToDevice, d.stream);
		}
		w->jointedPairsDirty = false;
	}
	checkCuda(w, "flush");
}

// RefreshBroadphase (reference src/world.cpp:156-229): fat boxes, active tier
// every call, stable tier when forced or dirty for >= 4 steps.
void refreshBroadphase(m3d_world* w, float dt)
{
	DevWorld& d = w->dev;
	int32_t n = (int32_t)w->bodies.size();
	bool rebuildStable = w->stableForce || (w->stableDirty && w->stepsSinceStableBuild >= 4);
	if (isBatch(w))
	{
		// each world on its own schedule (reference src/world.cpp:167-229)
		rebuildStable = false;
		const size_t worlds = w->batchRebuild.size();
		for (size_t k = 0; k < worlds; ++k)
		{
			const bool rb = w->batchStableForce[k] || (w->batchStableDirty[k] && w->batchStepsSinceStableBuild[k] >= 4);
			w->batchRebuild[k] = rb ? 1 : 0;
			rebuildStable |= rb;
			if (rb)
			{
				w->batchStableDirty[k] = 0;
				w->batchStableForce[k] = 0;
				w->batchStepsSinceStableBuild[k] = 0;
			}
			else
			{
				++w->batchStepsSinceStableBuild[k];
			}
		}
		cudaMemcpyAsync(d.worldRebuild.ptr, w->batchRebuild.data(), worlds, cudaMemcpyHostToDevice, d.stream);
	}
	w->lastRebuiltStable = rebuildStable;
	launchRefresh(d, n, dt, rebuildStable, w->def.gridCellSize);
	launchEmitGrid(d, n, w->def.gridCellSize, rebuildStable);
	readCounters(d); // sync: tier sizes and cell-key masks
	launchSortGrid(d, rebuildStable);
	if (rebuildStable)
	{
		w->stableDirty = false;
		w->stableForce = false;
		w->stepsSinceStableBuild = 0;
	}
	else
	{
		++w->stepsSinceStableBuild;
	}
	w->gridDirty = false;
}

// Events copied with the step's counters, before their counts are known: the
// first kEventHead entries of each list travel in the same round trip.
constexpr int32_t kEventHead = 1024;

// Pinned room for `need` events per list (contents are lost when it grows).
bool ensurePinnedEvents(m3d_world* w, int32_t need)
{
	if (need <= w->pinEventCap)
	{
		return false;
	}
	int32_t cap = w->pinEventCap * 2 > need ? w->pinEventCap * 2 : need;
	cap = cap < kEventHead ? kEventHead : cap;
	cudaFreeHost(w->pinEvents);
	cudaMallocHost((void**)&w->pinEvents, sizeof(int4) * 3 * (size_t)cap);
	w->pinEventCap = cap;
	return true;
}

// The step's last round trip: counters, the three event lists and (batch)
// the per-world stable-dirty words.  One stream wait, a second only when a
// list is longer than what travelled with the counters.  On return
// w->pinEvents + k * w->pinEventCap holds list k (removal ends, begins, ends).
void readStepResults(m3d_world* w)
{
	DevWorld& d = w->dev;
	cudaStream_t s = d.stream;
	ensurePinnedEvents(w, kEventHead);
	const DevBuf* lists[3] = { &d.evRemoval, &d.evBegin, &d.evEnd };
	int32_t copied[3];
	cudaMemcpyAsync(d.hostCounters, d.counters.ptr, sizeof(StepCounters), cudaMemcpyDeviceToHost, s);
	for (int k = 0; k < 3; ++k)
	{
		int64_t room = (int64_t)(lists[k]->bytes / sizeof(int4));
		copied[k] = (int32_t)(room < kEventHead ? room : kEventHead);
		if (copied[k] > 0)
		{
			cudaMemcpyAsync(w->pinEvents + (size_t)k * w->pinEventCap, lists[k]->ptr, sizeof(int4) * copied[k],
							cudaMemcpyDeviceToHost, s);
		}
	}
	if (isBatch(w))
	{
		if (d.worldCount > w->pinWorldDirtyCap)
		{
			cudaFreeHost(w->pinWorldDirty);
			cudaMallocHost((void**)&w->pinWorldDirty, sizeof(uint32_t) * (size_t)d.worldCount);
			w->pinWorldDirtyCap = d.worldCount;
		}
		cudaMemcpyAsync(w->pinWorldDirty, d.worldStableDirty.ptr, sizeof(uint32_t) * (size_t)d.worldCount,
						cudaMemcpyDeviceToHost, s);
	}
	cudaStreamSynchronize(s);
	const StepCounters* hc = d.hostCounters;
	const int32_t counts[3] = { (int32_t)hc->endRemoval, (int32_t)hc->beginNP, (int32_t)hc->endNP };
	if (counts[0] > copied[0] || counts[1] > copied[1] || counts[2] > copied[2])
	{
		int32_t need = counts[0] > counts[1] ? counts[0] : counts[1];
		need = need > counts[2] ? need : counts[2];
		if (ensurePinnedEvents(w, need))
		{
			copied[0] = copied[1] = copied[2] = 0;
		}
		for (int k = 0; k < 3; ++k)
		{
			if (counts[k] > copied[k])
			{
				cudaMemcpyAsync(w->pinEvents + (size_t)k * w->pinEventCap + copied[k],
								lists[k]->as<int4>() + copied[k], sizeof(int4) * (size_t)(counts[k] - copied[k]),
								cudaMemcpyDeviceToHost, s);
			}
		}
		cudaStreamSynchronize(s);
	}
}

} // namespace


// ---- online autotuning (m3d_gpu_autotune) -------------------------------------
// Candidates differ only in which kernel solves a serial island (one warp, or
// one thread for islands of a few contacts); every candidate gives the same
// results bit for bit, so trials run on the world's real steps.

static std::string tuneKey(m3d_world* w)
{
	int dev = 0;
	cudaGetDevice(&dev);
	cudaDeviceProp prop;
	std::string name = cudaGetDeviceProperties(&prop, dev) == cudaSuccess ? prop.name : "unknown";
	for (char& c : name)
	{
		c = c == ' ' ? '_' : c;
	}
	int lb = 0, lw = 0;
	for (size_t n = w->bodies.size(); n > 1; n >>= 1)
	{
		++lb;
	}
	for (size_t n = w->batchFirstBody.size(); n > 1; n >>= 1)
	{
		++lw;
	}
	char buf[160];
	snprintf(buf, sizeof(buf), "%s|bodies2^%d|worlds2^%d", name.c_str(), lb, lw);
	return buf;
}

static bool tuneCacheLookup(const std::string& key, int2* out)
{
	const char* path = getenv("M3D_AUTOTUNE_CACHE");
	FILE* f = path != nullptr ? fopen(path, "r") : nullptr;
	if (f == nullptr)
	{
		return false;
	}
	char k[200];
	int a = 0, b = 0;
	bool found = false;
	while (fscanf(f, "%199s %d %d", k, &a, &b) == 3)
	{
		if (key == k)
		{
			*out = make_int2(a, b); // the last entry for a key wins
			found = true;
		}
	}
	fclose(f);
	return found;
}

static void tuneCacheStore(const std::string& key, int2 v)
{
	const char* path = getenv("M3D_AUTOTUNE_CACHE");
	FILE* f = path != nullptr ? fopen(path, "a") : nullptr;
	if (f != nullptr)
	{
		fprintf(f, "%s %d %d\n", key.c_str(), v.x, v.y);
		fclose(f);
	}
}

static void tuneApply(m3d_world* w, int2 v)
{
	w->dev.tinyContacts = v.x;
	w->dev.tinyModeIslands = (uint32_t)v.y;
}

static void tuneBeforeStep(m3d_world* w)
{
	auto& t = w->tune;
	if (t.active)
	{
		tuneApply(w, t.candidates[(size_t)(t.step / t.stepsPerTrial) % t.candidates.size()]);
	}
}

static void tuneAfterStep(m3d_world* w)
{
	auto& t = w->tune;
	if (!t.active)
	{
		return;
	}
	const size_t idx = (size_t)(t.step / t.stepsPerTrial) % t.candidates.size();
	t.samples[idx].push_back(w->lastDeviceMs);
	++t.step;
	if (t.step < t.stepsPerTrial * (int32_t)t.candidates.size() * t.rounds)
	{
		return;
	}
	float best = 0.0f;
	for (size_t k = 0; k < t.candidates.size(); ++k)
	{
		std::vector<float> v = t.samples[k];
		std::sort(v.begin(), v.end());
		const float med = v[v.size() / 2];
		if (t.chosen < 0 || med < best)
		{
			best = med;
			t.chosen = (int32_t)k;
		}
	}
	tuneApply(w, t.candidates[(size_t)t.chosen]);
	t.active = false;
	t.done = true;
	tuneCacheStore(t.key, t.candidates[(size_t)t.chosen]);
}

// ---- fixed scratch of m3d_gpu_sphere_cast_noalloc --------------------------------
// One block of device memory in the library image, sized for worlds of up to
// kNoAllocCastSlots body slots: the result record, the two pick keys and one
// candidate record per body slot.  It is shared by every world and every call
// on a device and keeps the last call's contents.
constexpr int32_t kNoAllocCastSlots = 65536;
constexpr size_t kNoAllocCastBytes = 128 + kCastRecBytes * (size_t)(kNoAllocCastSlots + 1);
static __device__ __align__(256) unsigned char g_noAllocCastScratch[kNoAllocCastBytes];

constexpr int kNoAllocMaxDevices = 64;
static void* g_noAllocCastPtr[kNoAllocMaxDevices] = {};
static void* g_noAllocCastCtx[kNoAllocMaxDevices] = {};
static std::mutex g_noAllocCastMutex;

// The current CUDA context (driver handle), through the runtime's driver
// entry point so the library needs no link against libcuda; null if the
// driver cannot say.
static void* currentContext()
{
	typedef int (*CtxGetCurrent)(void**);
	static CtxGetCurrent fn = [] {
		void* p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
			q != cudaDriverEntryPointSuccess)
		{
			p = nullptr;
		}
		return (CtxGetCurrent)p;
	}();
	void* ctx = nullptr;
	if (fn == nullptr || fn(&ctx) != 0)
	{
		return nullptr;
	}
	return ctx;
}

// Device address of the scratch block on `device`, which must be current.
// Looked up on the first call per device and cached together with the
// context it belongs to; when the device's context has been torn down and
// recreated since (cudaDeviceReset, or a host framework resetting the
// primary context), the cached address is stale and is looked up again.
static cudaError_t noAllocCastScratch(int device, void** out)
{
	if (device < 0 || device >= kNoAllocMaxDevices)
	{
		return cudaErrorInvalidDevice;
	}
	std::lock_guard<std::mutex> lock(g_noAllocCastMutex);
	void* ctx = currentContext();
	if (g_noAllocCastPtr[device] == nullptr || ctx == nullptr || ctx != g_noAllocCastCtx[device])
	{
		void* ptr = nullptr;
		cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noAllocCastScratch);
		if (e != cudaSuccess)
		{
			return e;
		}
		g_noAllocCastPtr[device] = ptr;
		g_noAllocCastCtx[device] = ctx;
	}
	*out = g_noAllocCastPtr[device];
	return cudaSuccess;
}

extern "C"
{

m3d_world_def m3d_world_def_default(void)
{
	m3d_world_def def;
	def.gravity = m3d_v3(0.0f, -9.81f, 0.0f);
	def.workerCount = 1;
	def.positionIterations = 2;
	def.gridCellSize = 1.5f;
	def.enableSleep = true;
	return def;
}

m3d_body_def m3d_body_def_default(void)
{
	m3d_body_def def;
	memset(&def, 0, sizeof(def));
	def.type = M3D_BODY_STATIC;
	def.position = m3d_v3_zero();
	def.orientation = m3d_quat_identity();
	def.linearVelocity = m3d_v3_zero();
	def.angularVelocity = m3d_v3_zero();
	def.linearDamping = 0.0f;
	def.angularDamping = 0.05f;
	def.gravityScale = 1.0f;
	def.enableSleep = true;
	def.isAwake = true;
	def.userData = 0;
	return def;
}

m3d_shape_def m3d_shape_def_default(void)
{
	m3d_shape_def def;
	memset(&def, 0, sizeof(def));
	def.type = M3D_SHAPE_SPHERE;
	def.radius = 0.5f;
	def.halfHeight = 0.5f;
	def.halfExtents = m3d_v3(0.5f, 0.5f, 0.5f);
	def.density = 1000.0f;
	def.friction = 0.6f;
	def.restitution = 0.0f;
	def.rollingResistance = 0.02f;
	def.filter = m3d_filter_default();
	def.isSensor = false;
	return def;
}

m3d_hinge_joint_def m3d_hinge_joint_def_default(void)
{
	m3d_hinge_joint_def def;
	memset(&def, 0, sizeof(def));
	def.bodyA = m3d_body_id_null();
	def.bodyB = m3d_body_id_null();
	def.localAxisA = m3d_v3(0.0f, 1.0f, 0.0f);
	return def;
}

m3d_weld_joint_def m3d_weld_joint_def_default(void)
{
	m3d_weld_joint_def def;
	memset(&def, 0, sizeof(def));
	def.bodyA = m3d_body_id_null();
	def.bodyB = m3d_body_id_null();
	return def;
}

m3d_world* m3d_world_create(const m3d_world_def* def)
{
	int devCount = 0;
	if (cudaGetDeviceCount(&devCount) != cudaSuccess || devCount <= 0)
	{
		fprintf(stderr, "melon3d_gpu: no CUDA device available; the GPU world cannot be created\n");
		cudaGetLastError();
		return nullptr;
	}
	m3d_world* w = new (std::nothrow) m3d_world();
	if (w == nullptr)
	{
		return nullptr;
	}
	w->def = def != nullptr ? *def : m3d_world_def_default();
	if (w->def.workerCount < 1)
	{
		w->def.workerCount = 1;
	}
	if (w->def.gridCellSize <= 0.1f)
	{
		w->def.gridCellSize = 2.5f;
	}
	if (cudaStreamCreateWithFlags(&w->dev.stream, cudaStreamNonBlocking) != cudaSuccess ||
		cudaEventCreate(&w->evStart) != cudaSuccess || cudaEventCreate(&w->evStop) != cudaSuccess)
	{
		fprintf(stderr, "melon3d_gpu: CUDA stream creation failed\n");
		cudaGetLastError();
		delete w;
		return nullptr;
	}
	memset(&w->profile, 0, sizeof(w->profile));
	devCounters(w->dev);
	if (!growBodies(w->dev, 1024) || !growContacts(w->dev, 4096))
	{
		fprintf(stderr, "melon3d_gpu: initial device allocation failed\n");
		delete w;
		return nullptr;
	}
	return w;
}

void m3d_world_destroy(m3d_world* world)
{
	if (world == nullptr)
	{
		return;
	}
	DevWorld& d = world->dev;
	cudaStreamSynchronize(d.stream);
	if (world->tape != nullptr)
	{
		tapeDestroy(world->tape);
		world->tape = nullptr;
	}
	BodySoA& B = d.B;
	void* bp[] = { B.pos, B.rot, B.vel, B.angVel, B.prevPos, B.prevRot, B.prevVel, B.prevAngVel, B.massInv,
				   B.iw0, B.iw1, B.iw2, B.force, B.torque, B.sleep, B.state, B.cold, B.fatLo, B.fatHi,
				   B.hasFat, B.moved, B.isActive, B.isStable, B.inStableTier, B.inStableCells, B.bFlags };
	for (void* p : bp)
	{
		cudaFree(p);
	}
	ContactSoA& C = d.C;
	void* cp[] = { C.bodies, C.pointCount, C.flags, C.normal, C.mat, C.cachePosA, C.cacheRotA, C.cachePosB,
				   C.cacheRotB, C.pAnchorA, C.pAnchorB, C.pFricA, C.pFricB, C.pSlip, C.pRA, C.pRB, C.pJA, C.pJB };
	for (void* p : cp)
	{
		cudaFree(p);
	}
	ContactSoA& C2 = d.C2;
	void* cp2[] = { C2.bodies, C2.pointCount, C2.flags, C2.normal, C2.mat, C2.cachePosA, C2.cacheRotA, C2.cachePosB,
					C2.cacheRotB, C2.pAnchorA, C2.pAnchorB, C2.pFricA, C2.pFricB, C2.pSlip, C2.pRA, C2.pRB, C2.pJA,
					C2.pJB };
	for (void* p : cp2)
	{
		cudaFree(p);
	}
	DevBuf* bufs[] = { &d.joints, &d.jointedPairs, &d.inActiveCells, &d.inStableCells, &d.cellCountA, &d.cellCountS,
					   &d.overFlagA, &d.overFlagS, &d.label, &d.islandFlag, &d.colorMask, &d.matDirty, &d.sleepFirstNo,
					   &d.sleepMin, &d.bodyKeys, &d.bodyVals, &d.activeKeys, &d.activeVals, &d.stableKeys,
					   &d.stableVals, &d.activeOver, &d.stableOver, &d.runStarts, &d.runFlag, &d.runPairCount,
					   &d.pairKeys, &d.overFlag, &d.overScan, &d.existingSet, &d.newSet, &d.newSetPos, &d.keepFlag,
					   &d.newContactKeys, &d.removeFlag, &d.removeScan, &d.moveSrc, &d.adjCount, &d.adjStart, &d.adjList, &d.transition, &d.evBeginFlag,
					   &d.evEndFlag, &d.evBegin, &d.evEnd, &d.evRemoval, &d.contactKeys, &d.contactVals,
					   &d.jointKeys, &d.jointVals, &d.islandStartFlag, &d.islands, &d.islandKinds, &d.colorOf,
					   &d.colorOrder, &d.colorStart, &d.packetMax, &d.contactColor, &d.uploads, &d.counters,
					   &d.queryOut };
	for (DevBuf* b : bufs)
	{
		b->release();
	}
	d.prim.release();
	if (d.hostCounters != nullptr)
	{
		cudaFreeHost(d.hostCounters);
	}
	cudaFreeHost(world->pinPos);
	cudaFreeHost(world->pinRot);
	cudaFreeHost(world->pinVel);
	cudaFreeHost(world->pinAng);
	cudaFreeHost(world->pinState);
	cudaFreeHost(world->pinSleep);
	cudaFreeHost(world->cBodies);
	cudaFreeHost(world->cFlags);
	cudaFreeHost(world->adjStart);
	cudaFreeHost(world->adjList);
	cudaFreeHost(world->pinEvents);
	cudaFreeHost(world->pinWorldDirty);
	dropSidecar(world);
	if (world->sideStream != nullptr)
	{
		cudaStreamDestroy(world->sideStream);
		cudaEventDestroy(world->sideDone);
	}
	world->sidePrim.release();
	cudaFreeHost(world->pinSideState);
	cudaEventDestroy(world->evStart);
	cudaEventDestroy(world->evStop);
	cudaStreamDestroy(d.stream);
	delete world;
}

// ---- bodies ------------------------------------------------------------------

m3d_body_id m3d_body_create(m3d_world* world, const m3d_body_def* bodyDef, const m3d_shape_def* shapeDef)
{
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: %s is not available on a batch of worlds\n", __func__);
		return m3d_body_id_null();
	}
	int32_t index;
	if (!world->freeBodies.empty())
	{
		index = world->freeBodies.back();
		world->freeBodies.pop_back();
	}
	else
	{
		index = (int32_t)world->bodies.size();
		world->bodies.emplace_back();
		memset(&world->bodies[index], 0, sizeof(HostBody));
		world->bodies[index].generation = 1;
	}
	HostBody& b = world->bodies[index];
	uint32_t gen = b.generation;
	memset(&b, 0, sizeof(HostBody));
	b.generation = gen;
	b.inUse = true;
	b.cold.type = (int32_t)bodyDef->type;
	b.position = bodyDef->position;
	b.rotation = m3d_quat_normalize(bodyDef->orientation);
	b.linearVelocity = bodyDef->linearVelocity;
	b.angularVelocity = bodyDef->angularVelocity;
	b.cold.linearDamping = bodyDef->linearDamping;
	b.cold.angularDamping = bodyDef->angularDamping;
	b.cold.gravityScale = bodyDef->gravityScale;
	b.enableSleep = bodyDef->enableSleep && world->def.enableSleep;
	b.isAwake = bodyDef->type == M3D_BODY_STATIC ? false : bodyDef->isAwake;
	b.sleepTime = 0.0f;
	b.smoothedEnergy = 4.0f * kSleepEnergyThresh;
	b.userData = bodyDef->userData;
	b.cold.shape.type = (int32_t)shapeDef->type;
	b.cold.shape.radius = shapeDef->radius;
	b.cold.shape.halfHeight = shapeDef->halfHeight;
	b.cold.shape.he = v3(shapeDef->halfExtents.x, shapeDef->halfExtents.y, shapeDef->halfExtents.z);
	b.cold.friction = shapeDef->friction;
	b.cold.restitution = shapeDef->restitution;
	b.cold.rollingResistance = shapeDef->rollingResistance;
	b.cold.categoryBits = shapeDef->filter.categoryBits;
	b.cold.maskBits = shapeDef->filter.maskBits;
	b.cold.groupIndex = shapeDef->filter.groupIndex;
	b.isSensor = shapeDef->isSensor;
	computeMassProperties(b, shapeDef);
	updateInvInertiaWorld(b);
	markDirty(world, index, kUpAll);
	world->gridDirty = true;
	world->stableDirty = true;
	return makeId(world, index);
}

void m3d_body_destroy(m3d_world* world, m3d_body_id id)
{
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: %s is not available on a batch of worlds\n", __func__);
		return;
	}
	HostBody* b = getBody(world, id);
	if (b == nullptr)
	{
		return;
	}
	prepareDestroy(world);
	++world->destroysSinceStep;
	int32_t index = id.index;
	// The reference scans every contact in descending index order
	// (src/world.cpp:578-594).  Its matches never move before they are
	// reached (only non-matching survivors from the tail are swapped down),
	// so visiting this body's live contacts in descending current slot order
	// removes the same contacts in the same order.
	std::vector<int32_t> slots;
	if (index < world->adjBodies)
	{
		for (uint32_t k = world->adjStart[index]; k < world->adjStart[index + 1]; ++k)
		{
			int32_t p = world->cPos[world->adjList[k]];
			if (p >= 0)
			{
				slots.push_back(p);
			}
		}
	}
	std::sort(slots.begin(), slots.end(), [](int32_t a, int32_t c) { return a > c; });
	for (int32_t i : slots)
	{
		int2 ab = world->cBodies[i];
		int32_t other = ab.x == index ? ab.y : ab.x;
		uint8_t fl = world->cFlags[i];
		if (fl & kCFTouching)
		{
			if (!(fl & kCFSensor))
			{
				wakeBodyHost(world, other);
			}
			m3d_contact_event e;
			e.bodyA = makeId(world, ab.x);
			e.bodyB = makeId(world, ab.y);
			e.isSensor = (fl & kCFSensor) != 0;
			world->endEvents.push_back(e);
		}
		removeContactAt(world, i);
	}
	for (int32_t i = 0; i < (int32_t)world->joints.size(); ++i)
	{
		JointRec& j = world->joints[i];
		if (j.inUse && (j.bodyA == index || j.bodyB == index))
		{
			wakeBodyHost(world, j.bodyA == index ? j.bodyB : j.bodyA);
			j.inUse = 0;
			j.generation++;
			world->freeJoints.push_back(i);
			world->jointedPairsDirty = true;
			world->jointsDirty = true;
		}
	}
	b->isAwake = hostAwake(world, index); // the state uploaded for the freed slot keeps the device's awake bit
	b->inUse = false;
	b->generation++;
	world->freeBodies.push_back(index);
	markDirty(world, index, kUpState);
	world->gridDirty = true;
	world->stableDirty = true;
	world->stableForce = true;
}

bool m3d_body_is_valid(m3d_world* world, m3d_body_id id) { return getBody(world, id) != nullptr; }

m3d_vec3 m3d_body_position(m3d_world* world, m3d_body_id id)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	return b != nullptr ? b->position : m3d_v3_zero();
}

m3d_quat m3d_body_rotation(m3d_world* world, m3d_body_id id)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	return b != nullptr ? b->rotation : m3d_quat_identity();
}

m3d_transform m3d_body_transform(m3d_world* world, m3d_body_id id)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr)
	{
		return { m3d_v3_zero(), m3d_quat_identity() };
	}
	return { b->position, b->rotation };
}

void m3d_body_set_transform(m3d_world* world, m3d_body_id id, m3d_vec3 position, m3d_quat rotation)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr)
	{
		return;
	}
	b->position = position;
	b->rotation = m3d_quat_normalize(rotation);
	updateInvInertiaWorld(*b);
	markDirty(world, id.index, kUpPose | kUpIW | kUpFatReset);
	world->gridDirty = true;
	markStableDirty(world, id.index);
	wakeBodyHost(world, id.index);
}

m3d_vec3 m3d_body_linear_velocity(m3d_world* world, m3d_body_id id)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	return b != nullptr ? b->linearVelocity : m3d_v3_zero();
}

m3d_vec3 m3d_body_angular_velocity(m3d_world* world, m3d_body_id id)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	return b != nullptr ? b->angularVelocity : m3d_v3_zero();
}

void m3d_body_set_linear_velocity(m3d_world* world, m3d_body_id id, m3d_vec3 v)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr || b->cold.type == kStatic)
	{
		return;
	}
	b->linearVelocity = v;
	markDirty(world, id.index, kUpVel);
	wakeBodyHost(world, id.index);
}

void m3d_body_set_angular_velocity(m3d_world* world, m3d_body_id id, m3d_vec3 w)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr || b->cold.type == kStatic)
	{
		return;
	}
	b->angularVelocity = w;
	markDirty(world, id.index, kUpVel);
	wakeBodyHost(world, id.index);
}

void m3d_body_apply_impulse(m3d_world* world, m3d_body_id id, m3d_vec3 impulse, m3d_vec3 worldPoint)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr || b->cold.type != kDynamic)
	{
		return;
	}
	updateInvInertiaWorld(*b);
	b->linearVelocity = m3d_mul_add(b->linearVelocity, b->invMass, impulse);
	m3d_vec3 r = m3d_sub(worldPoint, b->position);
	b->angularVelocity = m3d_add(b->angularVelocity, m3d_mat3_mulv(&b->invInertiaWorld, m3d_cross(r, impulse)));
	markDirty(world, id.index, kUpVel | kUpIW);
	wakeBodyHost(world, id.index);
}

float m3d_body_mass(m3d_world* world, m3d_body_id id)
{
	HostBody* b = getBody(world, id);
	return b != nullptr ? b->mass : 0.0f;
}

bool m3d_body_is_awake(m3d_world* world, m3d_body_id id)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	return b != nullptr && b->isAwake;
}

void m3d_body_wake(m3d_world* world, m3d_body_id id)
{
	syncMirror(world);
	if (getBody(world, id) != nullptr)
	{
		wakeBodyHost(world, id.index);
	}
}

uint64_t m3d_body_user_data(m3d_world* world, m3d_body_id id)
{
	HostBody* b = getBody(world, id);
	return b != nullptr ? b->userData : 0;
}

void m3d_body_set_user_data(m3d_world* world, m3d_body_id id, uint64_t userData)
{
	HostBody* b = getBody(world, id);
	if (b != nullptr)
	{
		b->userData = userData;
	}
}

m3d_body_type m3d_body_get_type(m3d_world* world, m3d_body_id id)
{
	HostBody* b = getBody(world, id);
	return b != nullptr ? (m3d_body_type)b->cold.type : M3D_BODY_STATIC;
}

void m3d_body_apply_force(m3d_world* world, m3d_body_id id, m3d_vec3 force)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr || b->cold.type != kDynamic)
	{
		return;
	}
	b->force = m3d_add(b->force, force);
	world->anyForcesApplied = true;
	markDirty(world, id.index, kUpForce);
	wakeBodyHost(world, id.index);
}

void m3d_body_apply_force_at_point(m3d_world* world, m3d_body_id id, m3d_vec3 force, m3d_vec3 worldPoint)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr || b->cold.type != kDynamic)
	{
		return;
	}
	b->force = m3d_add(b->force, force);
	m3d_vec3 r = m3d_sub(worldPoint, b->position);
	b->torque = m3d_add(b->torque, m3d_cross(r, force));
	world->anyForcesApplied = true;
	markDirty(world, id.index, kUpForce);
	wakeBodyHost(world, id.index);
}

void m3d_body_apply_torque(m3d_world* world, m3d_body_id id, m3d_vec3 torque)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr || b->cold.type != kDynamic)
	{
		return;
	}
	b->torque = m3d_add(b->torque, torque);
	world->anyForcesApplied = true;
	markDirty(world, id.index, kUpForce);
	wakeBodyHost(world, id.index);
}

void m3d_body_apply_angular_impulse(m3d_world* world, m3d_body_id id, m3d_vec3 impulse)
{
	syncMirror(world);
	HostBody* b = getBody(world, id);
	if (b == nullptr || b->cold.type != kDynamic)
	{
		return;
	}
	updateInvInertiaWorld(*b);
	b->angularVelocity = m3d_add(b->angularVelocity, m3d_mat3_mulv(&b->invInertiaWorld, impulse));
	markDirty(world, id.index, kUpVel | kUpIW);
	wakeBodyHost(world, id.index);
}

float m3d_body_friction(m3d_world* world, m3d_body_id id)
{
	HostBody* b = getBody(world, id);
	return b != nullptr ? b->cold.friction : 0.0f;
}

void m3d_body_set_friction(m3d_world* world, m3d_body_id id, float friction)
{
	HostBody* b = getBody(world, id);
	if (b == nullptr)
	{
		return;
	}
	b->cold.friction = friction < 0.0f ? 0.0f : friction;
	markDirty(world, id.index, kUpCold);
	world->anyMaterialChange = true;
}

float m3d_body_restitution(m3d_world* world, m3d_body_id id)
{
	HostBody* b = getBody(world, id);
	return b != nullptr ? b->cold.restitution : 0.0f;
}

void m3d_body_set_restitution(m3d_world* world, m3d_body_id id, float restitution)
{
	HostBody* b = getBody(world, id);
	if (b == nullptr)
	{
		return;
	}
	b->cold.restitution = restitution < 0.0f ? 0.0f : restitution;
	markDirty(world, id.index, kUpCold);
	world->anyMaterialChange = true;
}

m3d_vec3 m3d_world_gravity(m3d_world* world) { return world->def.gravity; }
void m3d_world_set_gravity(m3d_world* world, m3d_vec3 gravity)
{
	world->def.gravity = gravity;
	world->quiescent = false;
}

// ---- joints (reference src/world.cpp:868-1075) ------------------------------

static m3d_joint_id allocateJoint(m3d_world* world, JointRec** out)
{
	int32_t index;
	if (!world->freeJoints.empty())
	{
		index = world->freeJoints.back();
		world->freeJoints.pop_back();
	}
	else
	{
		index = (int32_t)world->joints.size();
		world->joints.emplace_back();
		memset(&world->joints[index], 0, sizeof(JointRec));
		world->joints[index].generation = 1;
	}
	world->quiescent = false;
	JointRec& j = world->joints[index];
	uint32_t gen = j.generation;
	memset(&j, 0, sizeof(JointRec));
	j.generation = gen;
	j.inUse = 1;
	world->jointedPairsDirty = true;
	world->jointsDirty = true;
	*out = &j;
	return { index, gen };
}

static V3 hv(m3d_vec3 v) { return v3(v.x, v.y, v.z); }
static m3d_vec3 mv(V3 v) { return m3d_v3(v.x, v.y, v.z); }

m3d_joint_id m3d_joint_create_distance(m3d_world* world, const m3d_distance_joint_def* def)
{
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: %s is not available on a batch of worlds\n", __func__);
		return { -1, 0 };
	}
	syncMirror(world);
	HostBody* a = getBody(world, def->bodyA);
	HostBody* b = getBody(world, def->bodyB);
	if (a == nullptr || b == nullptr || def->bodyA.index == def->bodyB.index)
	{
		return { -1, 0 };
	}
	JointRec* j;
	m3d_joint_id id = allocateJoint(world, &j);
	j->type = kJointDistance;
	j->bodyA = def->bodyA.index;
	j->bodyB = def->bodyB.index;
	j->localAnchorA = hv(def->localAnchorA);
	j->localAnchorB = hv(def->localAnchorB);
	j->hertz = def->hertz;
	j->dampingRatio = def->dampingRatio;
	j->lambda = 0.0f;
	if (def->length > 0.0f)
	{
		j->length = def->length;
	}
	else
	{
		m3d_vec3 pA = m3d_transform_point({ a->position, a->rotation }, def->localAnchorA);
		m3d_vec3 pB = m3d_transform_point({ b->position, b->rotation }, def->localAnchorB);
		j->length = m3d_length(m3d_sub(pB, pA));
	}
	int32_t ja = j->bodyA, jb = j->bodyB;
	wakeBodyHost(world, ja);
	wakeBodyHost(world, jb);
	return id;
}

m3d_joint_id m3d_joint_create_ball(m3d_world* world, const m3d_ball_joint_def* def)
{
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: %s is not available on a batch of worlds\n", __func__);
		return { -1, 0 };
	}
	syncMirror(world);
	HostBody* a = getBody(world, def->bodyA);
	HostBody* b = getBody(world, def->bodyB);
	if (a == nullptr || b == nullptr || def->bodyA.index == def->bodyB.index)
	{
		return { -1, 0 };
	}
	JointRec* j;
	m3d_joint_id id = allocateJoint(world, &j);
	j->type = kJointBall;
	j->bodyA = def->bodyA.index;
	j->bodyB = def->bodyB.index;
	j->localAnchorA = hv(def->localAnchorA);
	j->localAnchorB = hv(def->localAnchorB);
	j->lambda = 0.0f;
	int32_t ja = j->bodyA, jb = j->bodyB;
	wakeBodyHost(world, ja);
	wakeBodyHost(world, jb);
	return id;
}

m3d_joint_id m3d_joint_create_hinge(m3d_world* world, const m3d_hinge_joint_def* def)
{
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: %s is not available on a batch of worlds\n", __func__);
		return { -1, 0 };
	}
	syncMirror(world);
	HostBody* a = getBody(world, def->bodyA);
	HostBody* b = getBody(world, def->bodyB);
	if (a == nullptr || b == nullptr || def->bodyA.index == def->bodyB.index)
	{
		return { -1, 0 };
	}
	JointRec* j;
	m3d_joint_id id = allocateJoint(world, &j);
	j->type = kJointHinge;
	j->bodyA = def->bodyA.index;
	j->bodyB = def->bodyB.index;
	j->localAnchorA = hv(def->localAnchorA);
	j->localAnchorB = hv(def->localAnchorB);
	m3d_vec3 axisA = m3d_normalize(def->localAxisA);
	if (m3d_length_sq(axisA) < 0.5f)
	{
		axisA = m3d_v3(0.0f, 1.0f, 0.0f);
	}
	j->localAxisA = hv(axisA);
	if (m3d_length_sq(def->localAxisB) > 0.5f)
	{
		j->localAxisB = hv(m3d_normalize(def->localAxisB));
	}
	else
	{
		m3d_vec3 axisWorld = m3d_rotate(a->rotation, axisA);
		j->localAxisB = hv(m3d_inv_rotate(b->rotation, axisWorld));
	}
	{
		m3d_vec3 axisWorld = m3d_rotate(a->rotation, axisA);
		m3d_vec3 pick = fabsf(axisWorld.x) < 0.9f ? m3d_v3(1.0f, 0.0f, 0.0f) : m3d_v3(0.0f, 1.0f, 0.0f);
		m3d_vec3 refWorld = m3d_normalize(m3d_cross(axisWorld, pick));
		j->localRefA = hv(m3d_inv_rotate(a->rotation, refWorld));
		j->localRefB = hv(m3d_inv_rotate(b->rotation, refWorld));
	}
	j->enableLimit = def->enableLimit ? 1 : 0;
	j->lowerAngle = def->lowerAngle;
	j->upperAngle = def->upperAngle;
	j->enableMotor = def->enableMotor ? 1 : 0;
	j->motorSpeed = def->motorSpeed;
	j->maxMotorTorque = def->maxMotorTorque;
	j->lambda = 0.0f;
	j->motorLambda = 0.0f;
	int32_t ja = j->bodyA, jb = j->bodyB;
	wakeBodyHost(world, ja);
	wakeBodyHost(world, jb);
	return id;
}

m3d_joint_id m3d_joint_create_weld(m3d_world* world, const m3d_weld_joint_def* def)
{
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: %s is not available on a batch of worlds\n", __func__);
		return { -1, 0 };
	}
	syncMirror(world);
	HostBody* a = getBody(world, def->bodyA);
	HostBody* b = getBody(world, def->bodyB);
	if (a == nullptr || b == nullptr || def->bodyA.index == def->bodyB.index)
	{
		return { -1, 0 };
	}
	JointRec* j;
	m3d_joint_id id = allocateJoint(world, &j);
	j->type = kJointWeld;
	j->bodyA = def->bodyA.index;
	j->bodyB = def->bodyB.index;
	j->localAnchorA = hv(def->localAnchorA);
	j->localAnchorB = hv(def->localAnchorB);
	m3d_quat rel = m3d_quat_normalize(m3d_quat_mul(m3d_quat_conj(a->rotation), b->rotation));
	j->relRot0 = q4(rel.x, rel.y, rel.z, rel.w);
	j->lambda = 0.0f;
	int32_t ja = j->bodyA, jb = j->bodyB;
	wakeBodyHost(world, ja);
	wakeBodyHost(world, jb);
	return id;
}

static JointRec* getJoint(m3d_world* world, m3d_joint_id id)
{
	if (id.index < 0 || id.index >= (int32_t)world->joints.size())
	{
		return nullptr;
	}
	JointRec& j = world->joints[id.index];
	if (!j.inUse || j.generation != id.generation)
	{
		return nullptr;
	}
	return &j;
}

float m3d_joint_hinge_angle(m3d_world* world, m3d_joint_id id)
{
	syncMirror(world);
	JointRec* j = getJoint(world, id);
	if (j == nullptr || j->type != kJointHinge)
	{
		return 0.0f;
	}
	const HostBody& a = world->bodies[j->bodyA];
	const HostBody& b = world->bodies[j->bodyB];
	// HingeAngle (reference src/m3d_internal.h:354-362) on the host copy of the poses
	m3d_vec3 axis = m3d_rotate(a.rotation, mv(j->localAxisA));
	m3d_vec3 refA = m3d_rotate(a.rotation, mv(j->localRefA));
	m3d_vec3 refB = m3d_rotate(b.rotation, mv(j->localRefB));
	float s = m3d_dot(axis, m3d_cross(refA, refB));
	float c = m3d_dot(refA, refB);
	return atan2f(s, c);
}

void m3d_joint_hinge_set_motor(m3d_world* world, m3d_joint_id id, bool enable, float motorSpeed, float maxMotorTorque)
{
	syncMirror(world);
	JointRec* j = getJoint(world, id);
	if (j == nullptr || j->type != kJointHinge)
	{
		return;
	}
	j->enableMotor = enable ? 1 : 0;
	j->motorSpeed = motorSpeed;
	j->maxMotorTorque = maxMotorTorque < 0.0f ? 0.0f : maxMotorTorque;
	world->jointsDirty = true;
	int32_t ja = j->bodyA, jb = j->bodyB;
	wakeBodyHost(world, ja);
	wakeBodyHost(world, jb);
}

void m3d_joint_destroy(m3d_world* world, m3d_joint_id id)
{
	syncMirror(world);
	JointRec* j = getJoint(world, id);
	if (j == nullptr)
	{
		return;
	}
	int32_t ja = j->bodyA, jb = j->bodyB;
	wakeBodyHost(world, ja);
	wakeBodyHost(world, jb);
	j->inUse = 0;
	j->generation++;
	world->freeJoints.push_back(id.index);
	world->jointedPairsDirty = true;
	world->jointsDirty = true;
}

// ---- queries -----------------------------------------------------------------

static m3d_ray_result toRayResult(m3d_world* world, const RayQueryOut& q)
{
	m3d_ray_result r;
	r.body = q.hit ? makeId(world, q.body) : m3d_body_id_null();
	r.point = m3d_v3(q.point[0], q.point[1], q.point[2]);
	r.normal = m3d_v3(q.normal[0], q.normal[1], q.normal[2]);
	r.fraction = q.fraction;
	r.hit = q.hit != 0;
	return r;
}

static m3d_ray_result noHit(m3d_world* world, m3d_vec3 origin, m3d_vec3 translation)
{
	RayQueryOut q;
	q.body = -1;
	q.hit = 0;
	q.fraction = 2.0f;
	m3d_vec3 end = m3d_add(origin, translation);
	q.point[0] = end.x;
	q.point[1] = end.y;
	q.point[2] = end.z;
	q.normal[0] = q.normal[1] = q.normal[2] = 0.0f;
	return toRayResult(world, q);
}

static m3d_ray_result rayCastInternal(m3d_world* world, m3d_vec3 origin, m3d_vec3 translation, uint32_t maskBits)
{
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: queries are not available on a batch of worlds\n");
		return noHit(world, origin, translation);
	}
	syncMirror(world);
	flushHostChanges(world);
	if (world->gridDirty || world->stableDirty)
	{
		refreshBroadphase(world, 0.0f);
	}
	RayQueryOut q;
	launchRayCast(world->dev, (int32_t)world->bodies.size(), hv(origin), hv(translation), maskBits,
				  world->def.gridCellSize, &q);
	checkCuda(world, "ray cast");
	return toRayResult(world, q);
}

m3d_ray_result m3d_world_ray_cast(m3d_world* world, m3d_vec3 origin, m3d_vec3 translation)
{
	return rayCastInternal(world, origin, translation, 0xFFFFFFFFu);
}

m3d_ray_result m3d_world_ray_cast_filtered(m3d_world* world, m3d_vec3 origin, m3d_vec3 translation, uint32_t maskBits)
{
	return rayCastInternal(world, origin, translation, maskBits);
}

m3d_ray_result m3d_world_sphere_cast(m3d_world* world, m3d_vec3 origin, float radius, m3d_vec3 translation,
									 uint32_t maskBits)
{
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: queries are not available on a batch of worlds\n");
		return noHit(world, origin, translation);
	}
	syncMirror(world);
	flushHostChanges(world);
	RayQueryOut q;
	launchSphereCast(world->dev, (int32_t)world->bodies.size(), hv(origin), radius, hv(translation), maskBits, &q);
	checkCuda(world, "sphere cast");
	return toRayResult(world, q);
}

void m3d_world_overlap_aabb(m3d_world* world, m3d_aabb aabb, m3d_overlap_fn fn, void* context)
{
	if (fn == NULL || isBatch(world))
	{
		return;
	}
	syncMirror(world);
	flushHostChanges(world);
	int32_t n = (int32_t)world->bodies.size();
	std::vector<uint8_t> flags((size_t)n + 1, 0);
	Box box;
	box.lo = hv(aabb.lowerBound);
	box.hi = hv(aabb.upperBound);
	launchOverlap(world->dev, n, box, flags.data());
	checkCuda(world, "overlap");
	for (int32_t i = 0; i < n; ++i)
	{
		if (flags[i] && !fn(makeId(world, i), context))
		{
			return;
		}
	}
}

m3d_contact_events m3d_world_contact_events(m3d_world* world)
{
	m3d_contact_events ev;
	ev.beginEvents = world->beginEvents.data();
	ev.beginCount = (int32_t)world->beginEvents.size();
	ev.endEvents = world->endEvents.data();
	ev.endCount = (int32_t)world->endEvents.size();
	return ev;
}

m3d_profile m3d_world_profile(m3d_world* world) { return world->profile; }

// ---- step ----------------------------------------------------------------------

void m3d_world_step(m3d_world* world, float dt, int substepCount)
{
	if (dt <= 0.0f)
	{
		return;
	}
	if (substepCount < 1)
	{
		substepCount = 1;
	}
	DevWorld& d = world->dev;
	auto tStart = Clock::now();
	dropSidecar(world);
	world->awakeBitsValid = false;
	const bool churned = world->destroysSinceStep > 0; // destroys since the last step
	world->destroysSinceStep = 0;
	world->beginEvents.clear();
	world->endEvents.clear();
	if (world->quiescent && world->tape == nullptr && !isBatch(world) && world->dirtyList.empty() &&
		!world->anyForcesApplied && !world->anyMaterialChange && !world->jointsDirty && !world->jointedPairsDirty &&
		!(world->contactMirrorValid && world->contactsEdited) && !world->gridDirty && !world->stableDirty &&
		!world->stableForce && world->status == M3D_GPU_OK)
	{
		// Sleeping-world fast path.  The last step changed nothing: every body
		// was asleep before and after it, it admitted, created and removed no
		// pair, saw no touch transition, did not rebuild the stable tier and
		// left it clean, and no API call has edited the world since.  The
		// reference's step on such a world refreshes no fat box, enumerates
		// nothing (the active tier is empty), skips every sleeping pair in the
		// narrowphase and takes the no-awake-body early-out
		// (src/world.cpp:1848-1862), so it changes nothing but its stable-tier
		// step count and profile: this step does the same on the host, with
		// no device work.
		++world->stepsSinceStableBuild;
		world->lastDeviceMs = 0.0f;
		auto tEnd = Clock::now();
		world->profile.broadphaseMs = toMs(tStart, tEnd);
		world->profile.narrowphaseMs = 0.0f;
		world->profile.solverMs = 0.0f;
		world->profile.stepMs = toMs(tStart, tEnd);
		world->profile.awakeBodyCount = 0;
		world->profile.touchingContactCount = 0;
		world->profile.islandCount = 0;
		++world->quiescentSteps;
		return;
	}
	tuneBeforeStep(world);
	cudaEventRecord(world->evStart, d.stream);
	const int32_t n = (int32_t)world->bodies.size();
	const bool editsAtStart = !world->dirtyList.empty() || world->anyForcesApplied || world->anyMaterialChange ||
							  world->jointsDirty || world->jointedPairsDirty ||
							  (world->contactMirrorValid && world->contactsEdited);

	if (world->tape != nullptr)
	{
		if (tapeSteps(world->tape) > 0 && !world->dirtyList.empty())
		{
			tapeMarkUnsupported(world->tape, "bodies were edited between recorded steps");
		}
		if (world->anyForcesApplied)
		{
			tapeMarkUnsupported(world->tape, "applied forces are not differentiated");
		}
	}
	flushHostChanges(world);
	StepCounters* dc = devCounters(d);
	resetStepCounters(d, (uint32_t)d.contactCount); // all zero but the contact count
	if (world->tape != nullptr)
	{
		tapeStepBegin(world->tape, d, n, dt, substepCount, hv(world->def.gravity), world->def.positionIterations);
	}
	if (isBatch(world))
	{
		fillWords(d.worldStableDirty.ptr, 0u, sizeof(uint32_t) * (size_t)d.worldCount, d.stream);
	}

	// broadphase and pair bookkeeping: sync 1 inside (tier sizes), sync 2
	// after counting the admitted pairs (buffer sizes)
	refreshBroadphase(world, dt);
	launchFindRuns(d);
	launchPairCount(d, n, world->def.gridCellSize);
	readCounters(d);
	if (d.hostCounters->hashFail != 0)
	{
		setError(world, M3D_GPU_ERR_HASH, "pair hash table overflow");
	}
	int64_t admitted = (int64_t)d.hostCounters->gridPairs + d.hostCounters->overPairs;
	if (!growContacts(d, (int32_t)(d.contactCount + admitted + 1)))
	{
		setError(world, M3D_GPU_ERR_ALLOC, "contact arena growth failed");
		return;
	}
	launchPairEmit(d, n, world->def.gridCellSize);
	launchCreateContacts(d);
	if (isBatch(world))
	{
		launchBatchRelayout(d); // per-world swap-remove, worlds packed again
	}
	else
	{
		launchRemoval(d);
	}
	checkCuda(world, "broadphase");
	auto tBroad = Clock::now();

	// narrowphase, islands, solve, sleep: no host round trip until the end
	launchNarrowphase(d, dt);
	launchAnyAwakeDynamic(d, n);
	auto tNarrow = Clock::now();
	d.contactColor.ensure((size_t)(d.contactCap + 1) * sizeof(int32_t));
	fillWords(d.contactColor.ptr, 0xFFFFFFFFu, (size_t)(d.contactMax + 1) * sizeof(int32_t), d.stream);
	if (world->tape != nullptr)
	{
		tapeBeforeIslands(world->tape, d, substepCount);
	}
	launchIslands(d, n);
	launchSolve(d, dt, substepCount, hv(world->def.gravity), world->def.positionIterations);
	launchSleep(d, dt);
	launchFinish(d, n, dt, world->anyForcesApplied);
	cudaEventRecord(world->evStop, d.stream);

	// sync 3: counters with the step's events
	readStepResults(world);
	const StepCounters* hc = d.hostCounters;
	if (hc->waitErrors != 0)
	{
		setError(world, M3D_GPU_ERR_WAIT, "a bounded device wait ran out during the step");
	}
	checkCuda(world, "step");
	if (world->tape != nullptr)
	{
		tapeStepEnd(world->tape, d, *hc);
		checkCuda(world, "tape");
	}
	if (isBatch(world))
	{
		for (int32_t k = 0; k < d.worldCount; ++k)
		{
			if (world->pinWorldDirty[k] != 0)
			{
				world->batchStableDirty[k] = 1;
			}
		}
	}
	world->stepped = true;
	auto toEvent = [&](const int4& e) {
		m3d_contact_event ev;
		ev.bodyA = makeId(world, e.x);
		ev.bodyB = makeId(world, e.y);
		ev.isSensor = e.z != 0;
		return ev;
	};
	const int4* evR = world->pinEvents;
	const int4* evB = world->pinEvents + world->pinEventCap;
	const int4* evE = world->pinEvents + 2 * (size_t)world->pinEventCap;
	for (uint32_t k = 0; k < hc->endRemoval; ++k)
	{
		world->endEvents.push_back(toEvent(evR[k]));
	}
	for (uint32_t k = 0; k < hc->beginNP; ++k)
	{
		world->beginEvents.push_back(toEvent(evB[k]));
	}
	for (uint32_t k = 0; k < hc->endNP; ++k)
	{
		world->endEvents.push_back(toEvent(evE[k]));
	}
	d.contactCount = (int32_t)hc->contactCount;
	d.lastSerialIslands = hc->serialIslands;
	if (hc->anyAwakeDynamic)
	{
		d.islandsBuiltFor = n;
	}
	if (hc->stableDirty)
	{
		world->stableDirty = true;
	}
	if (world->anyForcesApplied)
	{
		for (HostBody& b : world->bodies)
		{
			if (b.inUse && b.cold.type == kDynamic)
			{
				b.force = m3d_v3_zero();
				b.torque = m3d_v3_zero();
			}
		}
		world->anyForcesApplied = false;
	}
	cudaEventElapsedTime(&world->lastDeviceMs, world->evStart, world->evStop);
	tuneAfterStep(world);
	world->mirrorStale = true;
	world->awakeStale = true;
	world->contactMirrorValid = false;

	auto tEnd = Clock::now();
	world->profile.broadphaseMs = toMs(tStart, tBroad);
	world->profile.narrowphaseMs = toMs(tBroad, tNarrow);
	world->profile.solverMs = toMs(tNarrow, tEnd);
	world->profile.stepMs = toMs(tStart, tEnd);
	world->profile.bodyCount = (int32_t)hc->bodyCount;
	world->profile.awakeBodyCount = (int32_t)hc->awakeBodyCount;
	world->profile.contactCount = d.contactCount;
	world->profile.touchingContactCount = (int32_t)hc->touchingCount;
	world->profile.islandCount = (int32_t)hc->islandCount;
	// a no-op step on a sleeping world: the next one (without edits) takes the
	// fast path at the top of this function
	world->quiescent = !editsAtStart && !isBatch(world) && world->tape == nullptr && world->status == M3D_GPU_OK &&
					   hc->awakeBodyCount == 0 && hc->anyAwakeDynamic == 0 && hc->newContacts == 0 &&
					   hc->removed == 0 && hc->endRemoval == 0 && hc->beginNP == 0 && hc->endNP == 0 &&
					   hc->stableDirty == 0 && hc->gridPairs == 0 && hc->overPairs == 0 && !world->lastRebuiltStable &&
					   !world->stableDirty && !world->stableForce;
	if (churned && !isBatch(world) && world->tape == nullptr && world->status == M3D_GPU_OK)
	{
		prefetchSidecar(world);
	}
}

// ---- GPU extensions ------------------------------------------------------------

int32_t m3d_gpu_body_capacity(m3d_world* world) { return (int32_t)world->bodies.size(); }

void m3d_gpu_read_poses(m3d_world* world, float* positions, float* rotations, int32_t capacity)
{
	flushHostChanges(world);
	int32_t n = (int32_t)world->bodies.size();
	n = n < capacity ? n : capacity;
	if (n <= 0)
	{
		return;
	}
	ensurePinned(world, n);
	DevWorld& d = world->dev;
	if (positions != nullptr)
	{
		cudaMemcpyAsync(world->pinPos, d.B.pos, sizeof(float4) * n, cudaMemcpyDeviceToHost, d.stream);
	}
	if (rotations != nullptr)
	{
		cudaMemcpyAsync(world->pinRot, d.B.rot, sizeof(float4) * n, cudaMemcpyDeviceToHost, d.stream);
	}
	cudaStreamSynchronize(d.stream);
	if (positions != nullptr)
	{
		const float4* src = world->pinPos;
		for (int32_t i = 0; i < n; ++i)
		{
			positions[3 * i + 0] = src[i].x;
			positions[3 * i + 1] = src[i].y;
			positions[3 * i + 2] = src[i].z;
		}
	}
	if (rotations != nullptr)
	{
		memcpy(rotations, world->pinRot, sizeof(float4) * (size_t)n);
	}
}

float m3d_gpu_last_step_device_ms(m3d_world* world) { return world->lastDeviceMs; }

int32_t m3d_gpu_step_counters(m3d_world* world, uint32_t* out, int32_t capacity)
{
	const int32_t n = (int32_t)(sizeof(StepCounters) / sizeof(uint32_t));
	const uint32_t* src = (const uint32_t*)world->dev.hostCounters;
	for (int32_t i = 0; i < n && i < capacity && src != nullptr; ++i)
	{
		out[i] = src[i];
	}
	return n;
}
int32_t m3d_gpu_status(m3d_world* world) { return world->status; }

// ---- batch of worlds ----------------------------------------------------------

m3d_world* m3d_gpu_batch_create(m3d_world* const* worlds, int32_t count)
{
	if (worlds == nullptr || count < 1)
	{
		fprintf(stderr, "melon3d_gpu: m3d_gpu_batch_create: no worlds\n");
		return nullptr;
	}
	const m3d_world_def& def0 = worlds[0] != nullptr ? worlds[0]->def : m3d_world_def();
	for (int32_t k = 0; k < count; ++k)
	{
		const m3d_world* w = worlds[k];
		if (w == nullptr || w->stepped || isBatch(w))
		{
			fprintf(stderr, "melon3d_gpu: m3d_gpu_batch_create: world %d is missing, was already stepped or is a batch\n",
					k);
			return nullptr;
		}
		const m3d_world_def& d = w->def;
		if (d.gravity.x != def0.gravity.x || d.gravity.y != def0.gravity.y || d.gravity.z != def0.gravity.z ||
			d.positionIterations != def0.positionIterations || d.gridCellSize != def0.gridCellSize ||
			d.enableSleep != def0.enableSleep)
		{
			fprintf(stderr, "melon3d_gpu: m3d_gpu_batch_create: world %d has a different world definition\n", k);
			return nullptr;
		}
	}
	int worldBits = 0;
	while (worldBits < 31 && ((int64_t)1 << worldBits) < count)
	{
		++worldBits;
	}
	const int keyBits = (63 - worldBits) / 3;
	if (keyBits < 12)
	{
		fprintf(stderr, "melon3d_gpu: m3d_gpu_batch_create: %d worlds leave too few cell-key bits\n", count);
		return nullptr;
	}
	m3d_world_def def = def0;
	m3d_world* b = m3d_world_create(&def);
	if (b == nullptr)
	{
		return nullptr;
	}
	const int32_t worldCount = count;
	b->batchStableDirty.resize(worldCount);
	b->batchStableForce.resize(worldCount);
	b->batchStepsSinceStableBuild.resize(worldCount);
	b->batchRebuild.assign(worldCount, 0);
	for (int32_t k = 0; k < worldCount; ++k)
	{
		m3d_world* src = worlds[k];
		syncMirror(src);
		const int32_t base = (int32_t)b->bodies.size();
		b->batchFirstBody.push_back(base);
		for (const HostBody& hb : src->bodies)
		{
			b->bodies.push_back(hb);
			b->bodyWorld.push_back((uint32_t)k);
		}
		for (const JointRec& j : src->joints)
		{
			JointRec jr = j;
			jr.bodyA += base;
			jr.bodyB += base;
			b->joints.push_back(jr);
		}
		b->batchStableDirty[k] = src->stableDirty ? 1 : 0;
		b->batchStableForce[k] = src->stableForce ? 1 : 0;
		b->batchStepsSinceStableBuild[k] = src->stepsSinceStableBuild;
		b->anyForcesApplied |= src->anyForcesApplied;
		b->anyMaterialChange |= src->anyMaterialChange;
	}
	const int32_t n = (int32_t)b->bodies.size();
	b->batchFirstBody.push_back(n);
	for (int32_t i = 0; i < n; ++i)
	{
		markDirty(b, i, kUpAll);
	}
	b->jointsDirty = true;
	b->jointedPairsDirty = true;
	b->gridDirty = true;

	DevWorld& d = b->dev;
	d.batched = true;
	d.worldCount = worldCount;
	d.keyBits = keyBits;
	bool ok = growBodies(d, n + 1);
	ok = ok && d.worldOf.ensureZeroed(sizeof(uint32_t) * (size_t)d.bodyCap, d.stream);
	ok = ok && d.worldRebuild.ensureZeroed((size_t)worldCount + 1, d.stream);
	ok = ok && d.worldStableDirty.ensureZeroed(sizeof(uint32_t) * (size_t)(worldCount + 1), d.stream);
	ok = ok && d.worldContactCount.ensureZeroed(sizeof(uint32_t) * (size_t)(worldCount + 1), d.stream);
	ok = ok && d.worldContactStart.ensureZeroed(sizeof(uint32_t) * (size_t)(worldCount + 1), d.stream);
	ok = ok && d.worldFirstBody.ensure(sizeof(uint32_t) * (size_t)(worldCount + 1));
	if (ok && n > 0)
	{
		cudaMemcpyAsync(d.worldOf.ptr, b->bodyWorld.data(), sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice,
						d.stream);
	}
	if (ok)
	{
		cudaMemcpyAsync(d.worldFirstBody.ptr, b->batchFirstBody.data(), sizeof(uint32_t) * (size_t)(worldCount + 1),
						cudaMemcpyHostToDevice, d.stream);
	}
	for (int32_t k = 0; k < worldCount; ++k)
	{
		const int32_t nk = b->batchFirstBody[k + 1] - b->batchFirstBody[k];
		d.maxWorldBodies = nk > d.maxWorldBodies ? nk : d.maxWorldBodies;
	}
	d.B.world = d.worldOf.as<uint32_t>();
	// the second contact arena at the current capacity
	const int32_t cap = d.contactCap;
	d.contactCap = 0;
	ok = ok && growContacts(d, cap);
	cudaStreamSynchronize(d.stream);
	if (!ok || cudaGetLastError() != cudaSuccess)
	{
		fprintf(stderr, "melon3d_gpu: m3d_gpu_batch_create: device allocation failed\n");
		m3d_world_destroy(b);
		return nullptr;
	}
	return b;
}

int32_t m3d_gpu_batch_world_count(m3d_world* batch)
{
	return isBatch(batch) ? (int32_t)batch->batchFirstBody.size() - 1 : 1;
}

int32_t m3d_gpu_batch_first_body(m3d_world* batch, int32_t worldIndex)
{
	if (!isBatch(batch))
	{
		return worldIndex == 0 ? 0 : (worldIndex == 1 ? (int32_t)batch->bodies.size() : -1);
	}
	if (worldIndex < 0 || worldIndex >= (int32_t)batch->batchFirstBody.size())
	{
		return -1;
	}
	return batch->batchFirstBody[worldIndex];
}

void m3d_gpu_set_wait_limit(m3d_world* world, int64_t polls)
{
	world->dev.prim.waitLimit = polls < 0 ? -1 : polls;
}

void m3d_gpu_clear_status(m3d_world* world)
{
	world->status = M3D_GPU_OK;
	world->errorText[0] = 0;
}

int32_t m3d_gpu_autotune(m3d_world* world, int32_t stepsPerTrial)
{
	auto& t = world->tune;
	t = m3d_world::Tune();
	if (stepsPerTrial <= 0)
	{
		tuneApply(world, make_int2(kTinyIslandContacts, (int)kTinyModeIslands));
		return 0;
	}
	t.key = tuneKey(world);
	int2 cached;
	if (tuneCacheLookup(t.key, &cached))
	{
		tuneApply(world, cached);
		t.candidates.push_back(cached);
		t.chosen = 0;
		t.done = true;
		return 1;
	}
	// the default (tiny islands one thread each once a step has more than
	// 16384 serial islands), every serial island on a warp, and one thread for
	// islands of up to 2, 4, 8 or 16 contacts at any island count
	t.candidates = { make_int2(kTinyIslandContacts, (int)kTinyModeIslands), make_int2(0, 0), make_int2(2, 0),
					 make_int2(4, 0), make_int2(8, 0), make_int2(16, 0) };
	t.samples.assign(t.candidates.size(), std::vector<float>());
	t.stepsPerTrial = stepsPerTrial;
	t.rounds = 2;
	t.active = true;
	return 0;
}

int32_t m3d_gpu_autotune_state(m3d_world* world, int32_t* tinyContacts, int32_t* tinyModeIslands)
{
	if (tinyContacts != nullptr)
	{
		*tinyContacts = world->dev.tinyContacts;
	}
	if (tinyModeIslands != nullptr)
	{
		*tinyModeIslands = (int32_t)world->dev.tinyModeIslands;
	}
	return world->tune.active ? 1 : (world->tune.done ? 2 : 0);
}

int64_t m3d_gpu_fast_path_steps(m3d_world* world) { return world->quiescentSteps; }

int32_t m3d_gpu_giant_profile(m3d_world* world, double* out, int32_t capacity)
{
	DevWorld& d = world->dev;
	if (d.giantMisc.ptr == nullptr || out == nullptr || capacity <= 0)
	{
		return 0;
	}
	uint32_t misc[16];
	unsigned long long ns[16];
	cudaMemcpyAsync(misc, d.giantMisc.ptr, sizeof(misc), cudaMemcpyDeviceToHost, d.stream);
	cudaMemcpyAsync(ns, (const char*)d.giantMisc.ptr + sizeof(misc), sizeof(ns), cudaMemcpyDeviceToHost, d.stream);
	cudaStreamSynchronize(d.stream);
	int32_t ncol = 0;
	for (int c = 0; c < kMaxGraphColors; ++c)
	{
		ncol = misc[c + 1] > misc[c] ? c + 1 : ncol;
	}
	double v[15];
	for (int k = 0; k < 5; ++k)
	{
		v[k] = ns[k + 1] >= ns[k] ? (double)(ns[k + 1] - ns[k]) : 0.0;
	}
	v[5] = (double)ncol;
	v[6] = (double)misc[kMaxGraphColors + 4];
	v[7] = (double)misc[kMaxGraphColors + 3];
	for (int k = 0; k < 7; ++k)
	{
		v[8 + k] = (double)ns[8 + k];
	}
	int32_t n = capacity < 15 ? capacity : 15;
	for (int32_t k = 0; k < n; ++k)
	{
		out[k] = v[k];
	}
	return n;
}

void m3d_gpu_set_giant_island_contacts(m3d_world* world, int32_t contacts)
{
	world->dev.giantIslandContacts = contacts < kBigIslandContacts ? kBigIslandContacts : contacts;
}
const char* m3d_gpu_last_error_string(m3d_world* world) { return world->errorText; }

int32_t m3d_gpu_sphere_cast_noalloc(m3d_world* world, m3d_vec3 origin, float radius, m3d_vec3 translation,
									uint32_t maskBits, m3d_ray_result* out)
{
	if (world == nullptr || out == nullptr)
	{
		fprintf(stderr, "melon3d_gpu: m3d_gpu_sphere_cast_noalloc: world and out must not be NULL\n");
		return M3D_GPU_ERR_ARGUMENT;
	}
	if (isBatch(world))
	{
		fprintf(stderr, "melon3d_gpu: queries are not available on a batch of worlds\n");
		*out = noHit(world, origin, translation);
		return M3D_GPU_ERR_ARGUMENT;
	}
	RayQueryOut miss;
	miss.body = -1;
	miss.hit = 0;
	miss.fraction = 2.0f;
	m3d_vec3 end = m3d_add(origin, translation);
	miss.point[0] = end.x;
	miss.point[1] = end.y;
	miss.point[2] = end.z;
	miss.normal[0] = miss.normal[1] = miss.normal[2] = 0.0f;
	*out = toRayResult(world, miss);

	const int32_t n = (int32_t)world->bodies.size();
	if (n > kNoAllocCastSlots)
	{
		fprintf(stderr,
				"melon3d_gpu: m3d_gpu_sphere_cast_noalloc: the world has %d body slots; the fixed scratch holds %d\n", n,
				kNoAllocCastSlots);
		return M3D_GPU_ERR_LIMIT;
	}
	// edits made through the API since the last step or query must be uploaded
	// first, and uploading may grow device buffers
	if (!world->dirtyList.empty() || (world->contactMirrorValid && world->contactsEdited) ||
		world->anyMaterialChange || world->jointsDirty || world->jointedPairsDirty || n + 1 > world->dev.bodyCap)
	{
		fprintf(stderr, "melon3d_gpu: m3d_gpu_sphere_cast_noalloc: the world has edits not yet on the device; "
						"step it or run any other query first\n");
		return M3D_GPU_ERR_PENDING;
	}

	cudaPointerAttributes attr;
	int current = 0;
	if (cudaPointerGetAttributes(&attr, world->dev.B.state) != cudaSuccess || cudaGetDevice(&current) != cudaSuccess)
	{
		checkCuda(world, "sphere cast (fixed scratch): device lookup");
		return M3D_GPU_ERR_CUDA;
	}
	const bool switched = attr.device != current;
	if (switched && cudaSetDevice(attr.device) != cudaSuccess)
	{
		checkCuda(world, "sphere cast (fixed scratch): cudaSetDevice");
		return M3D_GPU_ERR_CUDA;
	}
	int32_t rc = M3D_GPU_OK;
	void* scratch = nullptr;
	cudaError_t e = noAllocCastScratch(attr.device, &scratch);
	if (e != cudaSuccess)
	{
		char buf[256];
		snprintf(buf, sizeof(buf), "sphere cast (fixed scratch): cudaGetSymbolAddress: %s", cudaGetErrorString(e));
		cudaGetLastError();
		setError(world, M3D_GPU_ERR_CUDA, buf);
		rc = M3D_GPU_ERR_CUDA;
	}
	else
	{
		RayQueryOut q;
		launchSphereCastInto(world->dev, n, hv(origin), radius, hv(translation), maskBits, scratch, &q);
		cudaError_t le = cudaGetLastError();
		if (le != cudaSuccess)
		{
			char buf[256];
			snprintf(buf, sizeof(buf), "sphere cast (fixed scratch): %s", cudaGetErrorString(le));
			setError(world, M3D_GPU_ERR_CUDA, buf);
			rc = M3D_GPU_ERR_CUDA;
		}
		else
		{
			*out = toRayResult(world, q);
		}
	}
	if (switched)
	{
		cudaSetDevice(current);
	}
	return rc;
}

// ---- snapshots (include/melon3d_debug.h) ----------------------------------------

int32_t m3d_dbg_body_capacity(m3d_world* world) { return (int32_t)world->bodies.size(); }

void m3d_dbg_bodies(m3d_world* world, m3d_dbg_body* out, int32_t capacity)
{
	flushHostChanges(world);
	int32_t n = (int32_t)world->bodies.size();
	n = n < capacity ? n : capacity;
	if (n <= 0)
	{
		return;
	}
	DevWorld& d = world->dev;
	std::vector<float4> pos(n), rot(n), vel(n), ang(n), ppos(n), prot(n), i0(n), i1(n), i2(n), flo(n), fhi(n);
	std::vector<float2> sl(n);
	std::vector<uint8_t> st(n), hf(n);
	cudaStream_t s = d.stream;
	cudaMemcpyAsync(pos.data(), d.B.pos, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(rot.data(), d.B.rot, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(vel.data(), d.B.vel, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(ang.data(), d.B.angVel, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(ppos.data(), d.B.prevPos, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(prot.data(), d.B.prevRot, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(i0.data(), d.B.iw0, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(i1.data(), d.B.iw1, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(i2.data(), d.B.iw2, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(flo.data(), d.B.fatLo, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(fhi.data(), d.B.fatHi, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(sl.data(), d.B.sleep, sizeof(float2) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(st.data(), d.B.state, n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(hf.data(), d.B.hasFat, n, cudaMemcpyDeviceToHost, s);
	cudaStreamSynchronize(s);
	for (int32_t i = 0; i < n; ++i)
	{
		m3d_dbg_body& o = out[i];
		memset(&o, 0, sizeof(o));
		float4 v4[] = { pos[i], vel[i], ang[i], ppos[i], i0[i], i1[i], i2[i], flo[i], fhi[i] };
		float* dst3[] = { o.position, o.linearVelocity, o.angularVelocity, o.prevPosition, o.invInertiaWorld,
						  o.invInertiaWorld + 3, o.invInertiaWorld + 6, o.fatLower, o.fatUpper };
		for (int k = 0; k < 9; ++k)
		{
			dst3[k][0] = v4[k].x;
			dst3[k][1] = v4[k].y;
			dst3[k][2] = v4[k].z;
		}
		o.rotation[0] = rot[i].x;
		o.rotation[1] = rot[i].y;
		o.rotation[2] = rot[i].z;
		o.rotation[3] = rot[i].w;
		o.prevRotation[0] = prot[i].x;
		o.prevRotation[1] = prot[i].y;
		o.prevRotation[2] = prot[i].z;
		o.prevRotation[3] = prot[i].w;
		o.sleepTime = sl[i].x;
		o.smoothedEnergy = sl[i].y;
		o.hasFatAABB = hf[i];
		o.isAwake = (st[i] & kStAwake) ? 1 : 0;
		o.inUse = (st[i] & kStInUse) ? 1 : 0;
	}
}

int32_t m3d_dbg_contact_count(m3d_world* world)
{
	flushHostChanges(world);
	return world->dev.contactCount;
}

void m3d_dbg_contacts(m3d_world* world, m3d_dbg_contact* out, int32_t capacity)
{
	flushHostChanges(world);
	DevWorld& d = world->dev;
	int32_t n = d.contactCount < capacity ? d.contactCount : capacity;
	if (n <= 0)
	{
		return;
	}
	int32_t cap = d.contactCap;
	std::vector<int2> bodies(n);
	std::vector<int32_t> pc(n);
	std::vector<uint8_t> fl(n);
	std::vector<float4> nrm(n);
	std::vector<float2> mat(n);
	std::vector<float4> pa(4 * (size_t)cap), pb(4 * (size_t)cap), fa(4 * (size_t)cap), fb(4 * (size_t)cap),
		ps(4 * (size_t)cap);
	cudaStream_t s = d.stream;
	cudaMemcpyAsync(bodies.data(), d.C.bodies, sizeof(int2) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(pc.data(), d.C.pointCount, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(fl.data(), d.C.flags, n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(nrm.data(), d.C.normal, sizeof(float4) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(mat.data(), d.C.mat, sizeof(float2) * n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(pa.data(), d.C.pAnchorA, sizeof(float4) * 4 * cap, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(pb.data(), d.C.pAnchorB, sizeof(float4) * 4 * cap, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(fa.data(), d.C.pFricA, sizeof(float4) * 4 * cap, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(fb.data(), d.C.pFricB, sizeof(float4) * 4 * cap, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(ps.data(), d.C.pSlip, sizeof(float4) * 4 * cap, cudaMemcpyDeviceToHost, s);
	cudaStreamSynchronize(s);
	for (int32_t c = 0; c < n; ++c)
	{
		m3d_dbg_contact& o = out[c];
		memset(&o, 0, sizeof(o));
		o.bodyA = bodies[c].x;
		o.bodyB = bodies[c].y;
		o.pointCount = pc[c];
		o.touching = (fl[c] & kCFTouching) ? 1 : 0;
		o.isSensor = (fl[c] & kCFSensor) ? 1 : 0;
		o.tunnelGuard = (fl[c] & kCFTunnelGuard) ? 1 : 0;
		o.hasCache = (fl[c] & kCFHasCache) ? 1 : 0;
		o.normal[0] = nrm[c].x;
		o.normal[1] = nrm[c].y;
		o.normal[2] = nrm[c].z;
		o.friction = nrm[c].w;
		o.restitution = mat[c].x;
		o.rollingResistance = mat[c].y;
		for (int32_t p = 0; p < pc[c] && p < 4; ++p)
		{
			size_t k = (size_t)p * cap + c;
			m3d_dbg_point& q = o.points[p];
			q.localAnchorA[0] = pa[k].x;
			q.localAnchorA[1] = pa[k].y;
			q.localAnchorA[2] = pa[k].z;
			q.separation = pa[k].w;
			q.localAnchorB[0] = pb[k].x;
			q.localAnchorB[1] = pb[k].y;
			q.localAnchorB[2] = pb[k].z;
			memcpy(&q.id, &pb[k].w, sizeof(uint32_t));
			q.frictionAnchorA[0] = fa[k].x;
			q.frictionAnchorA[1] = fa[k].y;
			q.frictionAnchorA[2] = fa[k].z;
			q.lambdaN = fa[k].w;
			q.frictionAnchorB[0] = fb[k].x;
			q.frictionAnchorB[1] = fb[k].y;
			q.frictionAnchorB[2] = fb[k].z;
			q.lambdaT = fb[k].w;
			q.slipDir[0] = ps[k].x;
			q.slipDir[1] = ps[k].y;
			q.slipDir[2] = ps[k].z;
			q.separationOffset = ps[k].w;
		}
	}
}

void m3d_dbg_island_labels(m3d_world* world, int32_t* out, int32_t capacity)
{
	DevWorld& d = world->dev;
	for (int32_t i = 0; i < capacity; ++i)
	{
		out[i] = -1;
	}
	if (d.label.ptr == nullptr || d.islandsBuiltFor <= 0)
	{
		return;
	}
	// every dynamic body's label (sleeping islands included) from the last
	// step that built islands, like the reference's persistent island lists
	int32_t n = d.islandsBuiltFor;
	n = n < capacity ? n : capacity;
	std::vector<int32_t> lab(n);
	cudaMemcpyAsync(lab.data(), d.label.ptr, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, d.stream);
	cudaStreamSynchronize(d.stream);
	for (int32_t i = 0; i < n; ++i)
	{
		out[i] = lab[i];
	}
}

void m3d_dbg_contact_colors(m3d_world* world, int32_t* out, int32_t capacity)
{
	DevWorld& d = world->dev;
	for (int32_t i = 0; i < capacity; ++i)
	{
		out[i] = -1;
	}
	int32_t n = d.contactCount < capacity ? d.contactCount : capacity;
	if (d.contactColor.ptr == nullptr || n <= 0)
	{
		return;
	}
	cudaMemcpyAsync(out, d.contactColor.ptr, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, d.stream);
	cudaStreamSynchronize(d.stream);
}

// ---- differentiation --------------------------------------------------------------

int32_t m3d_gpu_tape_begin(m3d_world* world, int32_t checkpointEvery)
{
	if (world == nullptr)
	{
		return M3D_GPU_ERR_ARGUMENT;
	}
	if (world->tape != nullptr)
	{
		tapeDestroy(world->tape);
		world->tape = nullptr;
	}
	flushHostChanges(world);
	world->tape = tapeCreate(world->dev, (int32_t)world->bodies.size(), checkpointEvery);
	checkCuda(world, "tape begin");
	return world->status;
}

void m3d_gpu_tape_end(m3d_world* world)
{
	if (world != nullptr && world->tape != nullptr)
	{
		cudaStreamSynchronize(world->dev.stream);
		tapeDestroy(world->tape);
		world->tape = nullptr;
	}
}

int64_t m3d_gpu_tape_warp_islands(m3d_world* world)
{
	return world != nullptr && world->tape != nullptr ? tapeWarpIslands(world->tape) : 0;
}

int64_t m3d_gpu_tape_bytes(m3d_world* world)
{
	return world != nullptr && world->tape != nullptr ? tapeBytes(world->tape) : 0;
}

int32_t m3d_gpu_tape_steps(m3d_world* world)
{
	return world != nullptr && world->tape != nullptr ? tapeSteps(world->tape) : 0;
}

int32_t m3d_gpu_tape_supported(m3d_world* world, char* why, int32_t capacity)
{
	const char* reason = world == nullptr || world->tape == nullptr ? "no tape is open" : tapeUnsupported(world->tape);
	if (why != nullptr && capacity > 0)
	{
		snprintf(why, (size_t)capacity, "%s", reason != nullptr ? reason : "");
	}
	return reason == nullptr ? 1 : 0;
}

static int32_t tapeUsable(m3d_world* world)
{
	if (world == nullptr || world->tape == nullptr)
	{
		return M3D_GPU_ERR_ARGUMENT;
	}
	if (tapeUnsupported(world->tape) != nullptr)
	{
		fprintf(stderr, "melon3d_gpu: tape not differentiable: %s\n", tapeUnsupported(world->tape));
		return M3D_GPU_ERR_UNSUPPORTED;
	}
	return tapeSteps(world->tape) > 0 ? M3D_GPU_OK : M3D_GPU_ERR_ARGUMENT;
}

int32_t m3d_gpu_tape_replay(m3d_world* world, float* positions, float* rotations, float* velocities,
							float* angularVelocities, int32_t capacity)
{
	int32_t rc = tapeUsable(world);
	if (rc != M3D_GPU_OK)
	{
		return rc;
	}
	rc = tapeReplay(world->tape, world->dev, positions, rotations, velocities, angularVelocities, capacity);
	checkCuda(world, "tape replay");
	return rc;
}

int32_t m3d_gpu_step_backward(m3d_world* world, const float* dPositions, const float* dRotations,
							  const float* dVelocities, const float* dAngularVelocities, float* gPositions,
							  float* gRotations, float* gVelocities, float* gAngularVelocities, float* gMass,
							  float* gFriction, float* gRestitution, int32_t capacity)
{
	int32_t rc = tapeUsable(world);
	if (rc != M3D_GPU_OK)
	{
		return rc;
	}
	rc = tapeBackward(world->tape, world->dev, dPositions, dRotations, dVelocities, dAngularVelocities, gPositions,
					  gRotations, gVelocities, gAngularVelocities, gMass, gFriction, gRestitution, capacity);
	checkCuda(world, "step backward");
	return rc;
}

int32_t m3d_gpu_step_backward_fp64_host(m3d_world* world, const double* dPositions, const double* dRotations,
										const double* dVelocities, const double* dAngularVelocities,
										double* gPositions, double* gRotations, double* gVelocities,
										double* gAngularVelocities, double* gMass, double* gFriction,
										double* gRestitution, int32_t capacity)
{
	int32_t rc = tapeUsable(world);
	if (rc != M3D_GPU_OK)
	{
		return rc;
	}
	return tapeBackwardHost(world->tape, dPositions, dRotations, dVelocities, dAngularVelocities, gPositions,
							gRotations, gVelocities, gAngularVelocities, gMass, gFriction, gRestitution, capacity);
}

int32_t m3d_gpu_tape_regenerate_host(m3d_world* world, int32_t doublePrecision, const double* dVelocities,
									 const double* dAngularVelocities, const double* dMass, const double* dFriction,
									 const double* dRestitution, double* positions, double* rotations,
									 double* velocities, double* angularVelocities, int32_t capacity)
{
	int32_t rc = tapeUsable(world);
	if (rc != M3D_GPU_OK)
	{
		return rc;
	}
	return tapeRegenerateHost(world->tape, doublePrecision, dVelocities, dAngularVelocities, dMass, dFriction,
							  dRestitution, positions, rotations, velocities, angularVelocities, capacity);
}

} // extern "C"

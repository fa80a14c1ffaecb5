// Differentiation of stepped trajectories: the tape recorded by
// m3d_world_step while a tape is open, the replay of recorded steps, the
// backward pass (m3d_gpu_step_backward), its FP64 host evaluation, and the
// regenerating replay that checks both - all through the differentiable
// substep of m3d_diff.h.
//
// Recorded per step: the islands that were solved (free and serial ones; a
// coloured island or a joint makes the tape unsupported), their body lists,
// for every substep the manifold of each island contact as contact
// preparation left it (with point ids and whether the narrowphase or the
// preparation regenerated it), each contact's position in the previous step
// (contact identity is the body pair), and the bodies put to sleep at the
// step's end.  Body states are checkpointed every `checkpointEvery` steps.
//
// Backward, segment by segment from the last checkpoint down: the segment's
// step-start states are recomputed by replaying the tape from its checkpoint
// (the replay reproduces the engine bit for bit), then each step is reversed
// in two launches, a recording forward (islandStepRecord) and the reverse
// (islandStepReverse).  Islands with many contacts get a warp each, whose
// lanes take the contacts of one dependency level at a time; the rest are
// packed one per thread (the island table is ordered by contact count when it
// is recorded).  The adjoint of every
// contact's manifold data travels with it from step to step (ContactBar,
// carried by the previous-position map) until the generation event that made
// it, where it turns into adjoints of the generation poses.  Sleeping at a
// step's end zeroes velocities, so their adjoints are cut there.
#include "m3d_dev.cuh"
#include "m3d_diff.h"
#include "melon3d_gpu.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <memory>
#include <vector>

namespace m3g
{

using m3d_diff::Body;
using m3d_diff::BodyConst;
using m3d_diff::IslandCtx;
using m3d_diff::TapeContact;
using m3d_diff::TapeIsland;

namespace
{

// device buffer that keeps its contents when it grows
struct GrowBuf
{
	DevBuf buf;
	size_t used = 0; // bytes
	bool reserve(size_t bytes, cudaStream_t s)
	{
		if (bytes <= buf.bytes && buf.ptr != nullptr)
		{
			return true;
		}
		size_t nb = buf.bytes * 2 > bytes ? buf.bytes * 2 : bytes;
		void* p = nullptr;
		countAllocation();
		if (cudaMalloc(&p, nb) != cudaSuccess)
		{
			return false;
		}
		if (buf.ptr != nullptr && used > 0)
		{
			cudaMemcpyAsync(p, buf.ptr, used, cudaMemcpyDeviceToDevice, s);
		}
		cudaStreamSynchronize(s);
		buf.release();
		buf.ptr = p;
		buf.bytes = nb;
		return true;
	}
	char* at(size_t offsetBytes) const { return (char*)buf.ptr + offsetBytes; }
};

// Contact records: bump-allocated in large device chunks that never move
// (a tape of a long trajectory holds gigabytes; growing one buffer by
// doubling would copy them over and over).
struct ChunkArena
{
	static constexpr size_t kChunkBytes = size_t(512) << 20;
	std::vector<std::unique_ptr<DevBuf>> chunks;
	size_t used = 0; // bytes used in the last chunk
	// room for `bytes` at the end of the last chunk (a new chunk if needed)
	char* reserve(size_t bytes)
	{
		if (chunks.empty() || used + bytes > chunks.back()->bytes)
		{
			std::unique_ptr<DevBuf> c(new DevBuf());
			if (!c->ensure(bytes > kChunkBytes ? bytes : kChunkBytes))
			{
				return nullptr;
			}
			chunks.push_back(std::move(c));
			used = 0;
		}
		return (char*)chunks.back()->ptr + used;
	}
	void commit(size_t bytes) { used += bytes; }
};

struct TapeStep
{
	size_t islandOff, bodyOff, sleepOff, posOff; // element offsets into the tape buffers
	const TapeContact* recs;                     // [substep * contactsPerSubstep + position]
	int32_t islands, bodies, contactsPerSubstep, sleeps;
	int32_t warpIslands; // islands [0, warpIslands) of the table are worked by a warp each
	float dt;
	int substeps, iterations;
	float g[3];
};

} // namespace

struct DiffTape
{
	int checkpointEvery = 10;
	int32_t nBodies = 0;
	int32_t warpContacts = 8; // islands with at least this many contacts get a warp in the replay and backward
	bool supported = true;
	char why[160] = { 0 };
	std::vector<TapeStep> steps;
	std::vector<int> checkpointStep; // step index of each checkpoint
	GrowBuf islands, bodies, sleeps, checkpoints;
	ChunkArena contacts;
	GrowBuf prevPos; // per step and contact position: the contact's position in the previous step, or -1
	DevBuf bodyConst, muBody, eBody, shapes, sleepScratch, flags;
	DevBuf hashKeys, hashVals; // body-pair key -> position in the previous step
	uint32_t hashMask = 0;
	DevBuf islandRaw, orderKeys, orderVals; // island table before it is ordered
	TapeStep pending;
};

void tapeMarkUnsupported(DiffTape* t, const char* why)
{
	if (t->supported)
	{
		t->supported = false;
		snprintf(t->why, sizeof(t->why), "%s", why);
	}
}

const char* tapeUnsupported(const DiffTape* t) { return t->supported ? nullptr : t->why; }

int32_t tapeSteps(const DiffTape* t) { return (int32_t)t->steps.size(); }

int64_t tapeWarpIslands(const DiffTape* t)
{
	int64_t n = 0;
	for (const TapeStep& st : t->steps)
	{
		n += st.warpIslands;
	}
	return n;
}

int64_t tapeBytes(const DiffTape* t)
{
	int64_t b = (int64_t)(t->islands.used + t->bodies.used + t->sleeps.used + t->checkpoints.used + t->prevPos.used);
	for (const TapeStep& st : t->steps)
	{
		b += (int64_t)st.contactsPerSubstep * st.substeps * (int64_t)sizeof(TapeContact);
	}
	return b;
}

void tapeDestroy(DiffTape* t) { delete t; }

// ---- recording -------------------------------------------------------------------

__global__ void kTapeBodyConst(BodySoA B, int32_t n, BodyConst<float>* bc, float* mu, float* e,
							   m3d_diff::TapeShape* shapes, uint32_t* bad)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	const BodyCold& c = B.cold[i];
	const float4 mi = B.massInv[i];
	const bool inUse = (B.state[i] & kStInUse) != 0;
	BodyConst<float> k;
	k.invMass = mi.x;
	k.il = mi.y;
	k.gravityScale = c.gravityScale;
	k.linearDamping = c.linearDamping;
	k.angularDamping = c.angularDamping;
	k.dynamic = inUse && c.type == kDynamic ? 1 : 0;
	bc[i] = k;
	mu[i] = c.friction;
	e[i] = c.restitution;
	m3d_diff::TapeShape sh;
	sh.type = c.shape.type;
	sh.radius = c.shape.radius;
	sh.he[0] = c.shape.he.x;
	sh.he[1] = c.shape.he.y;
	sh.he[2] = c.shape.he.z;
	shapes[i] = sh;
	if (inUse)
	{
		if (c.type == kKinematic)
		{
			atomicOr(bad, 1u);
		}
		if (c.shape.type == kCapsule)
		{
			atomicOr(bad, 2u);
		}
		if (k.dynamic && (mi.y != mi.z || mi.z != mi.w))
		{
			atomicOr(bad, 4u);
		}
	}
}

__global__ void kTapeCheckpoint(BodySoA B, int32_t n, Body<float>* out)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
	{
		return;
	}
	const float4 p = B.pos[i], q = B.rot[i], v = B.vel[i], w = B.angVel[i];
	Body<float> b;
	b.x = m3d_diff::v3<float>(p.x, p.y, p.z);
	b.q = m3d_diff::q4<float>(q.x, q.y, q.z, q.w);
	b.v = m3d_diff::v3<float>(v.x, v.y, v.z);
	b.w = m3d_diff::v3<float>(w.x, w.y, w.z);
	out[i] = b;
}

__global__ void kTapeIslands(const IslandRec* isl, const uint32_t* countDev, TapeIsland* out, uint32_t* bad)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= (int)*countDev)
	{
		return;
	}
	const IslandRec r = isl[k];
	TapeIsland t;
	t.bodyStart = r.bodyStart;
	t.bodyCount = r.bodyCount;
	t.contactStart = r.contactStart;
	t.contactCount = r.kind == 0 ? 0 : r.contactCount;
	out[k] = t;
	if (r.kind >= 2)
	{
		atomicOr(bad, 8u);
	}
	if (r.jointCount > 0)
	{
		atomicOr(bad, 16u);
	}
}

// Islands are independent (disjoint bodies and contacts, no sums across
// them), so the replay and the backward may take them in any order.  The
// table is ordered by falling contact count (then body count): the islands
// with at least `warpContacts` contacts form its head, each worked by a warp
// (its contacts level by level), and the rest are packed one per thread.
__global__ void kIslandWorkKeys(const TapeIsland* isl, int32_t n, int32_t warpContacts, uint64_t* keys,
								uint32_t* vals, uint32_t* warpCount)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < n)
	{
		const uint32_t c = (uint32_t)isl[k].contactCount, b = (uint32_t)isl[k].bodyCount;
		const uint64_t work = ((uint64_t)(c < 0xFFFFFu ? c : 0xFFFFFu) << 12) | (b < 0xFFFu ? b : 0xFFFu);
		keys[k] = 0xFFFFFFFFull - work;
		vals[k] = (uint32_t)k;
		if ((int32_t)c >= warpContacts)
		{
			atomicAdd(warpCount, 1u);
		}
	}
}

__global__ void kIslandGather(const TapeIsland* src, const uint32_t* order, int32_t n, TapeIsland* dst)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < n)
	{
		dst[k] = src[order[k]];
	}
}

// contact identity across steps: a contact is its body pair (the engine keeps
// one contact per pair, with a fixed body order)
constexpr unsigned long long kNoPairKey = ~0ull;

__device__ __forceinline__ unsigned long long pairKey(const TapeContact& c)
{
	return ((unsigned long long)(uint32_t)c.a << 32) | (unsigned long long)(uint32_t)c.b;
}
__device__ __forceinline__ uint32_t pairHash(unsigned long long k)
{
	k ^= k >> 33;
	k *= 0xff51afd7ed558ccdull;
	k ^= k >> 33;
	return (uint32_t)k;
}

// keys are unique within a step; the table holds at least twice as many
// slots as keys, so every probe sequence ends at an empty slot
__global__ void kPairInsert(const TapeContact* recs, int32_t n, unsigned long long* keys, int32_t* vals, uint32_t mask)
{
	M3G_KERNEL_BEGIN();
	int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n)
	{
		return;
	}
	const unsigned long long key = pairKey(recs[p]);
	uint32_t h = pairHash(key) & mask;
	for (uint32_t probe = 0; probe <= mask; ++probe)
	{
		const unsigned long long prev = atomicCAS(&keys[h], kNoPairKey, key);
		if (prev == kNoPairKey || prev == key)
		{
			vals[h] = p;
			return;
		}
		h = (h + 1) & mask;
	}
}

__global__ void kPairLookup(const TapeContact* recs, int32_t n, const unsigned long long* keys, const int32_t* vals,
							uint32_t mask, int32_t* out)
{
	M3G_KERNEL_BEGIN();
	int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n)
	{
		return;
	}
	const unsigned long long key = pairKey(recs[p]);
	uint32_t h = pairHash(key) & mask;
	int32_t found = -1;
	for (uint32_t probe = 0; probe <= mask; ++probe)
	{
		const unsigned long long k = keys[h];
		if (k == key)
		{
			found = vals[h];
			break;
		}
		if (k == kNoPairKey)
		{
			break;
		}
		h = (h + 1) & mask;
	}
	out[p] = found;
}

static void applyFlags(DiffTape* t, uint32_t flags)
{
	if (flags & 1u)
	{
		tapeMarkUnsupported(t, "kinematic bodies are not differentiated");
	}
	if (flags & 2u)
	{
		tapeMarkUnsupported(t, "capsules are not differentiated");
	}
	if (flags & 4u)
	{
		tapeMarkUnsupported(t, "a dynamic body has anisotropic inertia");
	}
	if (flags & 8u)
	{
		tapeMarkUnsupported(t, "an island of 300 or more contacts (coloured solve) is not differentiated");
	}
	if (flags & 16u)
	{
		tapeMarkUnsupported(t, "joints are not differentiated");
	}
}

DiffTape* tapeCreate(DevWorld& w, int32_t nBodies, int checkpointEvery)
{
	DiffTape* t = new DiffTape();
	t->checkpointEvery = checkpointEvery > 0 ? checkpointEvery : 10;
	t->nBodies = nBodies;
	if (const char* v = getenv("M3D_TAPE_WARP_CONTACTS"))
	{
		t->warpContacts = atoi(v) > 0 ? atoi(v) : 1 << 30;
	}
	const size_t n1 = (size_t)nBodies + 1;
	bool ok = t->bodyConst.ensure(sizeof(BodyConst<float>) * n1) && t->muBody.ensure(sizeof(float) * n1) &&
			  t->eBody.ensure(sizeof(float) * n1) && t->shapes.ensure(sizeof(m3d_diff::TapeShape) * n1) &&
			  t->sleepScratch.ensure(sizeof(uint32_t) * n1) && t->flags.ensure(sizeof(uint32_t) * 4);
	if (!ok)
	{
		tapeMarkUnsupported(t, "tape allocation failed");
		return t;
	}
	cudaMemsetAsync(t->flags.ptr, 0, sizeof(uint32_t) * 4, w.stream);
	if (nBodies > 0)
	{
		M3G_LAUNCH(kTapeBodyConst, blocksFor(nBodies, 256), 256, w.stream, w.B, nBodies,
				   t->bodyConst.as<BodyConst<float>>(), t->muBody.as<float>(), t->eBody.as<float>(),
				   t->shapes.as<m3d_diff::TapeShape>(), t->flags.as<uint32_t>());
	}
	uint32_t flags = 0;
	cudaMemcpyAsync(&flags, t->flags.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, w.stream);
	cudaStreamSynchronize(w.stream);
	applyFlags(t, flags);
	return t;
}

// At the start of a step (after host edits are on the device): checkpoint
// when due, and the step's constants.
void tapeStepBegin(DiffTape* t, DevWorld& w, int32_t n, float dt, int substeps, V3 g, int iterations)
{
	if (n != t->nBodies)
	{
		tapeMarkUnsupported(t, "bodies were created or destroyed while recording");
	}
	const int step = (int)t->steps.size();
	if (step % t->checkpointEvery == 0 && t->supported)
	{
		const size_t bytes = sizeof(Body<float>) * (size_t)t->nBodies;
		if (!t->checkpoints.reserve(t->checkpoints.used + bytes, w.stream))
		{
			tapeMarkUnsupported(t, "tape allocation failed");
		}
		else
		{
			if (t->nBodies > 0)
			{
				M3G_LAUNCH(kTapeCheckpoint, blocksFor(t->nBodies, 256), 256, w.stream, w.B, t->nBodies,
						   (Body<float>*)t->checkpoints.at(t->checkpoints.used));
			}
			t->checkpoints.used += bytes;
			t->checkpointStep.push_back(step);
		}
	}
	TapeStep& p = t->pending;
	memset(&p, 0, sizeof(p));
	p.dt = dt;
	p.substeps = substeps;
	p.iterations = iterations;
	p.g[0] = g.x;
	p.g[1] = g.y;
	p.g[2] = g.z;
	w.recording = true;
}

// Before the island build: room for this step's contact records (at most
// one per contact of the step and substep) and the sleep record.
void tapeBeforeIslands(DiffTape* t, DevWorld& w, int substeps)
{
	const size_t bound = (size_t)substeps * (size_t)(w.contactMax + 1);
	char* room = t->supported ? t->contacts.reserve(bound * sizeof(TapeContact)) : nullptr;
	if (room == nullptr)
	{
		tapeMarkUnsupported(t, "tape allocation failed");
		w.tapeContacts = nullptr;
		w.sleepRecord = nullptr;
		return;
	}
	w.tapeContacts = (TapeContact*)room;
	w.sleepRecord = t->sleepScratch.as<uint32_t>();
}

// After the step's last sync: the island table, the body list, the bodies put
// to sleep and each contact's position in the previous step go to the tape.
void tapeStepEnd(DiffTape* t, DevWorld& w, const StepCounters& hc)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	TapeStep st = t->pending;
	const bool solved = hc.anyAwakeDynamic != 0;
	st.islands = solved ? (int32_t)hc.awakeIslands : 0;
	st.bodies = solved ? (int32_t)hc.islandBodies : 0;
	st.contactsPerSubstep = solved ? (int32_t)hc.islandContacts : 0;
	st.sleeps = (int32_t)hc.sleptBodies;
	st.islandOff = t->islands.used / sizeof(TapeIsland);
	st.bodyOff = t->bodies.used / sizeof(int32_t);
	st.recs = w.tapeContacts;
	st.sleepOff = t->sleeps.used / sizeof(uint32_t);
	st.posOff = t->prevPos.used / sizeof(int32_t);
	if (hc.coloredIslands + hc.giantIslands > 0)
	{
		applyFlags(t, 8u);
	}
	if (hc.islandJoints > 0)
	{
		applyFlags(t, 16u);
	}
	if (w.tapeContacts == nullptr)
	{
		tapeMarkUnsupported(t, "tape allocation failed");
	}
	bool ok = t->supported &&
			  t->islands.reserve(t->islands.used + sizeof(TapeIsland) * (size_t)(st.islands + 1), s) &&
			  t->bodies.reserve(t->bodies.used + sizeof(int32_t) * (size_t)(st.bodies + 1), s) &&
			  t->sleeps.reserve(t->sleeps.used + sizeof(uint32_t) * (size_t)(st.sleeps + 1), s) &&
			  t->prevPos.reserve(t->prevPos.used + sizeof(int32_t) * (size_t)(st.contactsPerSubstep + 1), s);
	if (!ok)
	{
		tapeMarkUnsupported(t, "tape allocation failed");
	}
	else
	{
		if (st.islands > 0)
		{
			TapeIsland* out = (TapeIsland*)t->islands.at(t->islands.used);
			if (t->islandRaw.ensure(sizeof(TapeIsland) * (size_t)st.islands) &&
				t->orderKeys.ensure(sizeof(uint64_t) * (size_t)st.islands) &&
				t->orderVals.ensure(sizeof(uint32_t) * (size_t)st.islands))
			{
				TapeIsland* raw = t->islandRaw.as<TapeIsland>();
				M3G_LAUNCH(kTapeIslands, blocksFor(st.islands, 256), 256, s, w.islands.as<IslandRec>(),
						   &dc->awakeIslands, raw, t->flags.as<uint32_t>());
				cudaMemsetAsync(t->flags.as<uint32_t>() + 1, 0, sizeof(uint32_t), s);
				M3G_LAUNCH(kIslandWorkKeys, blocksFor(st.islands, 256), 256, s, raw, st.islands, t->warpContacts,
						   t->orderKeys.as<uint64_t>(), t->orderVals.as<uint32_t>(), t->flags.as<uint32_t>() + 1);
				radixSortPairs(t->orderKeys.as<uint64_t>(), t->orderVals.as<uint32_t>(), st.islands, 0xFFFFFFFFull,
							   w.prim, s);
				M3G_LAUNCH(kIslandGather, blocksFor(st.islands, 256), 256, s, raw, t->orderVals.as<uint32_t>(),
						   st.islands, out);
			}
			else
			{
				tapeMarkUnsupported(t, "tape allocation failed");
			}
			cudaMemcpyAsync(t->bodies.at(t->bodies.used), w.bodyVals.ptr, sizeof(int32_t) * (size_t)st.bodies,
							cudaMemcpyDeviceToDevice, s);
		}
		if (st.sleeps > 0)
		{
			cudaMemcpyAsync(t->sleeps.at(t->sleeps.used), w.sleepRecord, sizeof(uint32_t) * (size_t)st.sleeps,
							cudaMemcpyDeviceToDevice, s);
		}
		if (st.contactsPerSubstep > 0)
		{
			// each contact's position in the previous recorded step
			int32_t* out = (int32_t*)t->prevPos.at(t->prevPos.used);
			const TapeContact* cur = st.recs;
			const TapeStep* prev = t->steps.empty() ? nullptr : &t->steps.back();
			if (prev == nullptr || prev->contactsPerSubstep == 0)
			{
				cudaMemsetAsync(out, 0xFF, sizeof(int32_t) * (size_t)st.contactsPerSubstep, s);
			}
			else
			{
				uint32_t slots = 64;
				while (slots < 2u * (uint32_t)prev->contactsPerSubstep)
				{
					slots *= 2;
				}
				if (t->hashKeys.ensure(sizeof(unsigned long long) * slots) &&
					t->hashVals.ensure(sizeof(int32_t) * slots))
				{
					t->hashMask = slots - 1;
					cudaMemsetAsync(t->hashKeys.ptr, 0xFF, sizeof(unsigned long long) * slots, s);
					const TapeContact* before = prev->recs;
					M3G_LAUNCH(kPairInsert, blocksFor(prev->contactsPerSubstep, 256), 256, s, before,
							   prev->contactsPerSubstep, t->hashKeys.as<unsigned long long>(), t->hashVals.as<int32_t>(),
							   t->hashMask);
					M3G_LAUNCH(kPairLookup, blocksFor(st.contactsPerSubstep, 256), 256, s, cur, st.contactsPerSubstep,
							   t->hashKeys.as<unsigned long long>(), t->hashVals.as<int32_t>(), t->hashMask, out);
				}
				else
				{
					tapeMarkUnsupported(t, "tape allocation failed");
				}
			}
		}
		uint32_t flags[2] = { 0, 0 };
		cudaMemcpyAsync(flags, t->flags.ptr, sizeof(flags), cudaMemcpyDeviceToHost, s);
		cudaStreamSynchronize(s);
		applyFlags(t, flags[0]);
		st.warpIslands = st.islands > 0 ? (int32_t)flags[1] : 0;
		t->islands.used += sizeof(TapeIsland) * (size_t)st.islands;
		t->bodies.used += sizeof(int32_t) * (size_t)st.bodies;
		t->sleeps.used += sizeof(uint32_t) * (size_t)st.sleeps;
		t->prevPos.used += sizeof(int32_t) * (size_t)st.contactsPerSubstep;
		t->contacts.commit(sizeof(TapeContact) * (size_t)st.substeps * (size_t)st.contactsPerSubstep);
		t->steps.push_back(st);
	}
	w.recording = false;
	w.tapeContacts = nullptr;
	w.sleepRecord = nullptr;
}

// ---- replay and backward -------------------------------------------------------------

namespace
{

// work arrays of the replay / backward, host (double) or device (float)
template <typename T>
struct Work
{
	Body<T>* cur = nullptr;
	Body<T>* start = nullptr;
	m3d_diff::M<T>* iw = nullptr;
	m3d_diff::V<T>* x2 = nullptr;
	m3d_diff::Q<T>* q2 = nullptr;
	m3d_diff::Prepared<T>* prep = nullptr;
	T* lamN = nullptr;
	T* lamT = nullptr;
	m3d_diff::PoseRec<T>* normRec = nullptr;
	m3d_diff::PoseRec<T>* fricRec = nullptr;
	m3d_diff::VelRec<T>* velRec = nullptr;
	Body<T>* adj = nullptr;
	Body<T>* adj0 = nullptr;
	T* imBar = nullptr;
	T* ilBar = nullptr;
	T* muBar = nullptr;
	T* eBar = nullptr;
	m3d_diff::M<T>* iwBar = nullptr;
	m3d_diff::Prepared<T>* prepBar = nullptr;
	T* lamNBar = nullptr;
	T* lamTBar = nullptr;
	// dependency levels of a warp's island: per body the latest level, per
	// position the level, a level's count, and the positions by level
	int32_t* bodyLevel = nullptr;
	int32_t* levelOf = nullptr;
	int32_t* levelCount = nullptr;
	int32_t* order = nullptr;
	int32_t* orderLevel = nullptr;
	int32_t positions = 0;
};

struct Limits
{
	int maxSub = 1, maxIt = 1;
	int32_t positions = 1;
};

Limits tapeLimits(const DiffTape* t)
{
	Limits l;
	for (const TapeStep& st : t->steps)
	{
		l.maxSub = st.substeps > l.maxSub ? st.substeps : l.maxSub;
		l.maxIt = st.iterations > l.maxIt ? st.iterations : l.maxIt;
		l.positions = st.contactsPerSubstep > l.positions ? st.contactsPerSubstep : l.positions;
	}
	return l;
}

// carves the work arrays, zero-filled, out of an allocation function (device or host)
template <typename T, typename Alloc>
bool carveWork(Work<T>& k, int32_t n, const Limits& l, Alloc alloc)
{
	const size_t nb = (size_t)(n > 0 ? n : 1), np = (size_t)l.positions;
	k.positions = l.positions;
	k.cur = (Body<T>*)alloc(sizeof(Body<T>) * nb);
	k.start = (Body<T>*)alloc(sizeof(Body<T>) * nb * (size_t)l.maxSub);
	// per-substep records: one slice per substep (see substepView)
	const size_t S = (size_t)l.maxSub;
	k.iw = (m3d_diff::M<T>*)alloc(sizeof(m3d_diff::M<T>) * nb * S);
	k.x2 = (m3d_diff::V<T>*)alloc(sizeof(m3d_diff::V<T>) * nb * S);
	k.q2 = (m3d_diff::Q<T>*)alloc(sizeof(m3d_diff::Q<T>) * nb * S);
	k.prep = (m3d_diff::Prepared<T>*)alloc(sizeof(m3d_diff::Prepared<T>) * np * S);
	k.lamN = (T*)alloc(sizeof(T) * 4 * np * S);
	k.lamT = (T*)alloc(sizeof(T) * 4 * np * S);
	k.normRec = (m3d_diff::PoseRec<T>*)alloc(sizeof(m3d_diff::PoseRec<T>) * np * (size_t)l.maxIt * S);
	k.fricRec = (m3d_diff::PoseRec<T>*)alloc(sizeof(m3d_diff::PoseRec<T>) * np * S);
	k.velRec = (m3d_diff::VelRec<T>*)alloc(sizeof(m3d_diff::VelRec<T>) * np * S);
	k.adj = (Body<T>*)alloc(sizeof(Body<T>) * nb);
	k.adj0 = (Body<T>*)alloc(sizeof(Body<T>) * nb);
	k.imBar = (T*)alloc(sizeof(T) * nb);
	k.ilBar = (T*)alloc(sizeof(T) * nb);
	k.muBar = (T*)alloc(sizeof(T) * nb);
	k.eBar = (T*)alloc(sizeof(T) * nb);
	k.iwBar = (m3d_diff::M<T>*)alloc(sizeof(m3d_diff::M<T>) * nb);
	k.prepBar = (m3d_diff::Prepared<T>*)alloc(sizeof(m3d_diff::Prepared<T>) * np);
	k.lamNBar = (T*)alloc(sizeof(T) * 4 * np);
	k.lamTBar = (T*)alloc(sizeof(T) * 4 * np);
	k.bodyLevel = (int32_t*)alloc(sizeof(int32_t) * nb);
	k.levelOf = (int32_t*)alloc(sizeof(int32_t) * np);
	k.levelCount = (int32_t*)alloc(sizeof(int32_t) * np);
	k.order = (int32_t*)alloc(sizeof(int32_t) * np);
	k.orderLevel = (int32_t*)alloc(sizeof(int32_t) * np);
	return k.orderLevel != nullptr && k.lamTBar != nullptr && k.cur != nullptr && k.start != nullptr && k.normRec != nullptr;
}

// device allocations of one replay / backward call, freed together; each is
// zeroed on the call's stream, so the zeroing is ordered before the call's
// copies and kernels (the world's stream does not synchronise with the
// legacy default stream, where a plain cudaMemset would run)
struct DevArena
{
	cudaStream_t stream;
	explicit DevArena(cudaStream_t s) : stream(s) {}
	std::vector<void*> owned;
	bool ok = true;
	void* operator()(size_t bytes)
	{
		void* p = nullptr;
		countAllocation();
		if (cudaMalloc(&p, bytes) != cudaSuccess)
		{
			ok = false;
			return nullptr;
		}
		if (cudaMemsetAsync(p, 0, bytes, stream) != cudaSuccess)
		{
			ok = false;
		}
		owned.push_back(p);
		return p;
	}
	~DevArena()
	{
		for (void* p : owned)
		{
			cudaFree(p);
		}
	}
};

struct HostArena
{
	std::vector<std::vector<double>> owned;
	void* operator()(size_t bytes)
	{
		owned.emplace_back((bytes + sizeof(double) - 1) / sizeof(double), 0.0);
		return owned.back().data();
	}
};

template <typename T>
IslandCtx<T> makeCtx(const Work<T>& k, const BodyConst<T>* bc, const T* mu, const T* e, const TapeStep& st,
					 const TapeIsland* islands, const int32_t* bodies, const TapeContact* contacts, int32_t nBodies,
					 m3d_diff::ContactBar<T>* cbar = nullptr, const m3d_diff::TapeShape* shapes = nullptr,
					 const TapeContact* prevContacts = nullptr, const int32_t* prevPos = nullptr)
{
	IslandCtx<T> x;
	x.lane = 0;
	x.width = 1;
	x.order = nullptr;
	x.orderLevel = nullptr;
	x.genJ = nullptr;
	x.live = nullptr;
	x.liveIds = nullptr;
	x.cbar = cbar;
	x.shapes = shapes;
	x.prevContacts = prevContacts;
	x.prevPos = prevPos;
	x.dt = T(st.dt);
	x.bc = bc;
	x.h = T(st.dt) / T(st.substeps);
	x.invH = x.h > T(0) ? T(1) / x.h : T(0);
	x.maxCorrection = T(kMaxDepenetrationSpeed) * x.h;
	x.g = m3d_diff::v3<T>(T(st.g[0]), T(st.g[1]), T(st.g[2]));
	x.gravityLen = m3d_diff::len(x.g);
	x.iterations = st.iterations;
	x.substeps = st.substeps;
	x.island = islands;
	x.bodies = bodies;
	x.contacts = contacts;
	x.contactsPerSubstep = st.contactsPerSubstep;
	x.cur = k.cur;
	x.start = k.start;
	x.bodyCount = nBodies;
	x.iw = k.iw;
	x.x2 = k.x2;
	x.q2 = k.q2;
	x.prep = k.prep;
	x.lamN = k.lamN;
	x.lamT = k.lamT;
	x.normRec = k.normRec;
	x.fricRec = k.fricRec;
	x.velRec = k.velRec;
	x.positions = k.positions;
	x.adj = k.adj;
	x.adj0 = k.adj0;
	x.imBar = k.imBar;
	x.ilBar = k.ilBar;
	x.muBar = k.muBar;
	x.eBar = k.eBar;
	x.iwBar = k.iwBar;
	x.prepBar = k.prepBar;
	x.lamNBar = k.lamNBar;
	x.lamTBar = k.lamTBar;
	x.muBody = mu;
	x.eBody = e;
	return x;
}

} // namespace

// Dependency levels of the island's contacts (lane 0, then the warp
// synchronises): each contact one level above the latest earlier contact that
// shares a dynamic body with it; then the positions stably sorted by level.
// The body pair of a position is the same in every substep of the step.
__device__ void islandLevels(IslandCtx<float>& x, const Work<float>& k)
{
	const TapeIsland& r = *x.island;
	if (x.lane == 0)
	{
		for (int b = 0; b < r.bodyCount; ++b)
		{
			k.bodyLevel[x.bodies[r.bodyStart + b]] = -1;
		}
		int top = -1;
		for (int j = 0; j < r.contactCount; ++j)
		{
			const int pos = r.contactStart + j;
			const int a = x.contacts[pos].a, b = x.contacts[pos].b;
			const bool da = x.bc[a].dynamic != 0, db = x.bc[b].dynamic != 0;
			const int la = da ? k.bodyLevel[a] : -1, lb = db ? k.bodyLevel[b] : -1;
			const int level = (la > lb ? la : lb) + 1;
			k.levelOf[pos] = level;
			if (da)
			{
				k.bodyLevel[a] = level;
			}
			if (db)
			{
				k.bodyLevel[b] = level;
			}
			top = level > top ? level : top;
		}
		for (int l = 0; l <= top; ++l)
		{
			k.levelCount[r.contactStart + l] = 0;
		}
		for (int j = 0; j < r.contactCount; ++j)
		{
			k.levelCount[r.contactStart + k.levelOf[r.contactStart + j]] += 1;
		}
		int sum = 0;
		for (int l = 0; l <= top; ++l)
		{
			const int c = k.levelCount[r.contactStart + l];
			k.levelCount[r.contactStart + l] = sum;
			sum += c;
		}
		for (int j = 0; j < r.contactCount; ++j)
		{
			const int pos = r.contactStart + j;
			const int level = k.levelOf[pos];
			const int d = k.levelCount[r.contactStart + level]++;
			k.order[r.contactStart + d] = pos;
			k.orderLevel[r.contactStart + d] = level;
		}
	}
	__syncwarp();
	x.order = k.order;
	x.orderLevel = k.orderLevel;
}

// The island of this thread (one thread per island) or of this warp (the
// head of the table, warpIslands islands, one warp each, two per block);
// false when there is none.
__device__ bool islandOfThread(IslandCtx<float>& x, const IslandCtx<float>& base, const Work<float>& k,
							   int32_t islands, int32_t warpIslands)
{
	const int warpBlocks = (warpIslands + 1) / 2;
	x = base;
	if ((int)blockIdx.x < warpBlocks)
	{
		const int i = (int)blockIdx.x * 2 + (int)(threadIdx.x >> 5);
		if (i >= warpIslands)
		{
			return false; // the whole warp
		}
		x.island = base.island + i;
		x.lane = (int)(threadIdx.x & 31);
		x.width = 32;
		islandLevels(x, k);
		return true;
	}
	const int i = warpIslands + ((int)blockIdx.x - warpBlocks) * (int)blockDim.x + (int)threadIdx.x;
	if (i >= islands)
	{
		return false;
	}
	x.island = base.island + i;
	return true;
}

int32_t islandBlocks(const TapeStep& st)
{
	return (st.warpIslands + 1) / 2 + (int32_t)blocksFor(st.islands - st.warpIslands, 64);
}

__global__ void __launch_bounds__(64) kTapeReplayStep(IslandCtx<float> base, Work<float> k, int32_t islands,
													   int32_t warpIslands)
{
	M3G_KERNEL_BEGIN();
	IslandCtx<float> x;
	if (islandOfThread(x, base, k, islands, warpIslands))
	{
		m3d_diff::islandStepForward(x);
	}
}

__global__ void __launch_bounds__(64) kTapeRecordStep(IslandCtx<float> base, Work<float> k, int32_t islands,
													  int32_t warpIslands)
{
	M3G_KERNEL_BEGIN();
	IslandCtx<float> x;
	if (islandOfThread(x, base, k, islands, warpIslands))
	{
		m3d_diff::islandStepRecord(x);
	}
}

__global__ void __launch_bounds__(64) kTapeReverseStep(IslandCtx<float> base, Work<float> k, int32_t islands,
													   int32_t warpIslands)
{
	M3G_KERNEL_BEGIN();
	IslandCtx<float> x;
	if (islandOfThread(x, base, k, islands, warpIslands))
	{
		m3d_diff::islandStepReverse(x);
	}
}

// bodies put to sleep at a step's end: velocities (or their adjoints) zeroed
__global__ void kTapeSleepCut(Body<float>* b, const uint32_t* list, int32_t n)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < n)
	{
		b[list[k]].v = m3d_diff::vzero<float>();
		b[list[k]].w = m3d_diff::vzero<float>();
	}
}

// The Jacobians of the step's narrowphase generations, seven threads per
// contact (two columns each), at the step-start states (all the generations
// that happen at the step's start; those in contact preparation are evaluated
// by the island's own thread).
__global__ void __launch_bounds__(128)
	kTapeGenJacobian(const TapeContact* recs, int32_t n, const Body<float>* states, const BodyConst<float>* bc,
					 const m3d_diff::TapeShape* shapes, float dt, double* J)
{
	M3G_KERNEL_BEGIN();
	const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	const int64_t p = t / 7; // seven threads per contact, two Jacobian columns each
	if (p >= n)
	{
		return;
	}
	const TapeContact& rec = recs[p];
	if (!(rec.gen & m3d_diff::kTapeGenNarrow) || (rec.gen & m3d_diff::kTapeGenPrepare))
	{
		return;
	}
	const Body<float>& A = states[rec.a];
	const Body<float>& B = states[rec.b];
	const float margin = m3d_diff::kGenSpeculativeBase + dt * m3d_diff::len(m3d_diff::sub(A.v, B.v));
	m3d_diff::generationJacobianPair(bc, shapes, rec, A.x, A.q, B.x, B.q, margin, (int)(t % 7),
									 J + (size_t)p * (m3d_diff::kGenJRows * m3d_diff::kGenJCols));
}

// manifold adjoints carried to the previous step: contact p of this step is
// contact prevPos[p] there (or new)
__global__ void kTapeCarryBar(const m3d_diff::ContactBar<float>* cur, const int32_t* prevPos, int32_t n,
							  m3d_diff::ContactBar<float>* prev)
{
	M3G_KERNEL_BEGIN();
	int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p < n && prevPos[p] >= 0)
	{
		prev[prevPos[p]] = cur[p];
	}
}

namespace
{

IslandCtx<float> deviceCtx(DiffTape* t, const Work<float>& k, const TapeStep& st)
{
	return makeCtx<float>(k, t->bodyConst.as<BodyConst<float>>(), t->muBody.as<float>(), t->eBody.as<float>(), st,
						  (const TapeIsland*)t->islands.at(st.islandOff * sizeof(TapeIsland)),
						  (const int32_t*)t->bodies.at(st.bodyOff * sizeof(int32_t)),
						  st.recs, t->nBodies);
}

// the records of step `step - 1` at its last substep (null when it has none)
const TapeContact* previousRecords(const DiffTape* t, int step)
{
	if (step <= 0 || t->steps[step - 1].contactsPerSubstep == 0)
	{
		return nullptr;
	}
	const TapeStep& p = t->steps[step - 1];
	return p.recs + (size_t)(p.substeps - 1) * (size_t)p.contactsPerSubstep;
}

// replay steps [s0, s1) from the state in k.cur; the start state of each step
// goes to states[step - s0] when states is given
void replaySteps(DiffTape* t, cudaStream_t s, Work<float>& k, int s0, int s1, Body<float>* states)
{
	const int32_t n = t->nBodies;
	for (int step = s0; step < s1; ++step)
	{
		const TapeStep& st = t->steps[step];
		if (states != nullptr)
		{
			cudaMemcpyAsync(states + (size_t)(step - s0) * n, k.cur, sizeof(Body<float>) * (size_t)n,
							cudaMemcpyDeviceToDevice, s);
		}
		if (st.islands > 0)
		{
			M3G_LAUNCH(kTapeReplayStep, islandBlocks(st), 64, s, deviceCtx(t, k, st), k, st.islands, st.warpIslands);
		}
		if (st.sleeps > 0)
		{
			M3G_LAUNCH(kTapeSleepCut, blocksFor(st.sleeps, 256), 256, s, k.cur,
					   (const uint32_t*)t->sleeps.at(st.sleepOff * sizeof(uint32_t)), st.sleeps);
		}
	}
}

template <typename T, typename S>
void unpackBodies(const Body<T>* b, int32_t n, S* pos, S* rot, S* vel, S* ang)
{
	for (int32_t i = 0; i < n; ++i)
	{
		if (pos != nullptr)
		{
			pos[3 * i + 0] = (S)b[i].x.x;
			pos[3 * i + 1] = (S)b[i].x.y;
			pos[3 * i + 2] = (S)b[i].x.z;
		}
		if (rot != nullptr)
		{
			rot[4 * i + 0] = (S)b[i].q.x;
			rot[4 * i + 1] = (S)b[i].q.y;
			rot[4 * i + 2] = (S)b[i].q.z;
			rot[4 * i + 3] = (S)b[i].q.w;
		}
		if (vel != nullptr)
		{
			vel[3 * i + 0] = (S)b[i].v.x;
			vel[3 * i + 1] = (S)b[i].v.y;
			vel[3 * i + 2] = (S)b[i].v.z;
		}
		if (ang != nullptr)
		{
			ang[3 * i + 0] = (S)b[i].w.x;
			ang[3 * i + 1] = (S)b[i].w.y;
			ang[3 * i + 2] = (S)b[i].w.z;
		}
	}
}

template <typename T, typename S>
void packBodies(Body<T>* b, int32_t n, const S* pos, const S* rot, const S* vel, const S* ang)
{
	for (int32_t i = 0; i < n; ++i)
	{
		b[i].x = pos ? m3d_diff::v3<T>(T(pos[3 * i]), T(pos[3 * i + 1]), T(pos[3 * i + 2])) : m3d_diff::vzero<T>();
		b[i].q = rot ? m3d_diff::q4<T>(T(rot[4 * i]), T(rot[4 * i + 1]), T(rot[4 * i + 2]), T(rot[4 * i + 3]))
					 : m3d_diff::qzero<T>();
		b[i].v = vel ? m3d_diff::v3<T>(T(vel[3 * i]), T(vel[3 * i + 1]), T(vel[3 * i + 2])) : m3d_diff::vzero<T>();
		b[i].w = ang ? m3d_diff::v3<T>(T(ang[3 * i]), T(ang[3 * i + 1]), T(ang[3 * i + 2])) : m3d_diff::vzero<T>();
	}
}

// mass gradient: inertia scales with mass at fixed shape, so
// dL/dm = -invMass * (dL/dinvMass * invMass + dL/dil * il)
template <typename S>
S massGrad(const BodyConst<float>& c, S imBar, S ilBar)
{
	if (!c.dynamic || c.invMass <= 0.0f)
	{
		return S(0);
	}
	return -S(c.invMass) * (imBar * S(c.invMass) + ilBar * S(c.il));
}

} // namespace

int32_t tapeReplay(DiffTape* t, DevWorld& w, float* pos, float* rot, float* vel, float* angVel, int32_t capacity)
{
	if (t->steps.empty() || t->checkpointStep.empty())
	{
		return M3D_GPU_ERR_ARGUMENT;
	}
	const int32_t n = t->nBodies;
	DevArena arena(w.stream);
	Work<float> k;
	if (!carveWork(k, n, tapeLimits(t), [&](size_t b) { return arena(b); }) || !arena.ok)
	{
		return M3D_GPU_ERR_ALLOC;
	}
	cudaStream_t s = w.stream;
	cudaMemcpyAsync(k.cur, t->checkpoints.at(0), sizeof(Body<float>) * (size_t)n, cudaMemcpyDeviceToDevice, s);
	replaySteps(t, s, k, 0, (int)t->steps.size(), nullptr);
	std::vector<Body<float>> out((size_t)n);
	cudaMemcpyAsync(out.data(), k.cur, sizeof(Body<float>) * (size_t)n, cudaMemcpyDeviceToHost, s);
	cudaStreamSynchronize(s);
	if (cudaGetLastError() != cudaSuccess)
	{
		return M3D_GPU_ERR_CUDA;
	}
	unpackBodies(out.data(), n < capacity ? n : capacity, pos, rot, vel, angVel);
	return M3D_GPU_OK;
}

int32_t tapeBackward(DiffTape* t, DevWorld& w, const float* dPos, const float* dRot, const float* dVel,
					 const float* dAngVel, float* gPos, float* gRot, float* gVel, float* gAngVel, float* gMass,
					 float* gFriction, float* gRestitution, int32_t capacity)
{
	if (t->steps.empty() || t->checkpointStep.empty())
	{
		return M3D_GPU_ERR_ARGUMENT;
	}
	const int32_t n = t->nBodies;
	DevArena arena(w.stream);
	Work<float> k;
	const Limits lim = tapeLimits(t);
	bool ok = carveWork(k, n, lim, [&](size_t b) { return arena(b); });
	Body<float>* states = (Body<float>*)arena(sizeof(Body<float>) * (size_t)t->checkpointEvery * (size_t)(n + 1));
	typedef m3d_diff::ContactBar<float> Bar;
	Bar* bars[2] = { (Bar*)arena(sizeof(Bar) * (size_t)lim.positions), (Bar*)arena(sizeof(Bar) * (size_t)lim.positions) };
	const size_t jPer = (size_t)m3d_diff::kGenJRows * m3d_diff::kGenJCols;
	double* genJ = (double*)arena(sizeof(double) * jPer * (size_t)lim.positions);
	int cur = 0;
	if (!ok || !arena.ok)
	{
		return M3D_GPU_ERR_ALLOC;
	}
	cudaStream_t s = w.stream;
	{
		std::vector<Body<float>> seed((size_t)n);
		packBodies(seed.data(), n, dPos, dRot, dVel, dAngVel);
		cudaMemcpyAsync(k.adj, seed.data(), sizeof(Body<float>) * (size_t)n, cudaMemcpyHostToDevice, s);
		cudaStreamSynchronize(s);
	}
	const int S = (int)t->steps.size();
	for (int c = (int)t->checkpointStep.size() - 1; c >= 0; --c)
	{
		const int s0 = t->checkpointStep[c];
		const int s1 = c + 1 < (int)t->checkpointStep.size() ? t->checkpointStep[c + 1] : S;
		cudaMemcpyAsync(k.cur, t->checkpoints.at(sizeof(Body<float>) * (size_t)c * n), sizeof(Body<float>) * (size_t)n,
						cudaMemcpyDeviceToDevice, s);
		replaySteps(t, s, k, s0, s1, states);
		for (int step = s1 - 1; step >= s0; --step)
		{
			const TapeStep& st = t->steps[step];
			if (st.sleeps > 0)
			{
				M3G_LAUNCH(kTapeSleepCut, blocksFor(st.sleeps, 256), 256, s, k.adj,
						   (const uint32_t*)t->sleeps.at(st.sleepOff * sizeof(uint32_t)), st.sleeps);
			}
			const int32_t* prevPos =
				st.contactsPerSubstep > 0 ? (const int32_t*)t->prevPos.at(st.posOff * sizeof(int32_t)) : nullptr;
			if (st.islands > 0)
			{
				cudaMemcpyAsync(k.cur, states + (size_t)(step - s0) * n, sizeof(Body<float>) * (size_t)n,
								cudaMemcpyDeviceToDevice, s);
				if (st.contactsPerSubstep > 0)
				{
					M3G_LAUNCH(kTapeGenJacobian, blocksFor((int64_t)st.contactsPerSubstep * 7, 128), 128, s, st.recs,
							   st.contactsPerSubstep, states + (size_t)(step - s0) * n,
							   t->bodyConst.as<BodyConst<float>>(), t->shapes.as<m3d_diff::TapeShape>(), st.dt, genJ);
				}
				IslandCtx<float> x = deviceCtx(t, k, st);
				x.genJ = genJ;
				x.cbar = bars[cur];
				x.shapes = t->shapes.as<m3d_diff::TapeShape>();
				x.prevContacts = previousRecords(t, step);
				x.prevPos = prevPos;
				M3G_LAUNCH(kTapeRecordStep, islandBlocks(st), 64, s, x, k, st.islands, st.warpIslands);
				M3G_LAUNCH(kTapeReverseStep, islandBlocks(st), 64, s, x, k, st.islands, st.warpIslands);
			}
			if (step > 0)
			{
				// the manifold adjoints, carried to the contacts of the step before
				const TapeStep& pst = t->steps[step - 1];
				if (pst.contactsPerSubstep > 0)
				{
					cudaMemsetAsync(bars[1 - cur], 0, sizeof(Bar) * (size_t)pst.contactsPerSubstep, s);
					if (st.contactsPerSubstep > 0)
					{
						M3G_LAUNCH(kTapeCarryBar, blocksFor(st.contactsPerSubstep, 256), 256, s, bars[cur], prevPos,
								   st.contactsPerSubstep, bars[1 - cur]);
					}
				}
				cur = 1 - cur;
			}
		}
	}
	std::vector<Body<float>> adj((size_t)n);
	std::vector<float> im((size_t)n), il((size_t)n), mu((size_t)n), e((size_t)n);
	std::vector<BodyConst<float>> bc((size_t)n);
	cudaMemcpyAsync(adj.data(), k.adj, sizeof(Body<float>) * (size_t)n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(im.data(), k.imBar, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(il.data(), k.ilBar, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(mu.data(), k.muBar, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(e.data(), k.eBar, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s);
	cudaMemcpyAsync(bc.data(), t->bodyConst.ptr, sizeof(BodyConst<float>) * (size_t)n, cudaMemcpyDeviceToHost, s);
	cudaStreamSynchronize(s);
	if (cudaGetLastError() != cudaSuccess)
	{
		return M3D_GPU_ERR_CUDA;
	}
	const int32_t m = n < capacity ? n : capacity;
	unpackBodies(adj.data(), m, gPos, gRot, gVel, gAngVel);
	for (int32_t i = 0; i < m; ++i)
	{
		if (gMass != nullptr)
		{
			gMass[i] = massGrad<float>(bc[i], im[i], il[i]);
		}
		if (gFriction != nullptr)
		{
			gFriction[i] = mu[i];
		}
		if (gRestitution != nullptr)
		{
			gRestitution[i] = e[i];
		}
	}
	return M3D_GPU_OK;
}

// ---- host evaluations: the tape on the host ------------------------------------------

namespace
{
template <typename U>
std::vector<U> download(const GrowBuf& g, size_t offsetBytes, size_t count)
{
	std::vector<U> v(count);
	if (count > 0)
	{
		cudaMemcpy(v.data(), g.at(offsetBytes), sizeof(U) * count, cudaMemcpyDeviceToHost);
	}
	return v;
}

struct HostStep
{
	std::vector<TapeIsland> islands;
	std::vector<int32_t> bodies;
	std::vector<TapeContact> contacts;
	std::vector<uint32_t> sleeps;
	std::vector<int32_t> prevPos;
};

std::vector<HostStep> downloadSteps(const DiffTape* t)
{
	std::vector<HostStep> hs(t->steps.size());
	for (size_t q = 0; q < t->steps.size(); ++q)
	{
		const TapeStep& st = t->steps[q];
		hs[q].islands = download<TapeIsland>(t->islands, st.islandOff * sizeof(TapeIsland), (size_t)st.islands);
		hs[q].bodies = download<int32_t>(t->bodies, st.bodyOff * sizeof(int32_t), (size_t)st.bodies);
		hs[q].contacts.resize((size_t)st.substeps * (size_t)st.contactsPerSubstep);
		if (!hs[q].contacts.empty())
		{
			cudaMemcpy(hs[q].contacts.data(), st.recs, sizeof(TapeContact) * hs[q].contacts.size(),
					   cudaMemcpyDeviceToHost);
		}
		hs[q].sleeps = download<uint32_t>(t->sleeps, st.sleepOff * sizeof(uint32_t), (size_t)st.sleeps);
		hs[q].prevPos = download<int32_t>(t->prevPos, st.posOff * sizeof(int32_t), (size_t)st.contactsPerSubstep);
	}
	return hs;
}
} // namespace

// The same adjoint in double precision on the host, from the same tape.
int32_t tapeBackwardHost(DiffTape* t, const double* dPos, const double* dRot, const double* dVel,
						 const double* dAngVel, double* gPos, double* gRot, double* gVel, double* gAngVel,
						 double* gMass, double* gFriction, double* gRestitution, int32_t capacity)
{
	if (t->steps.empty() || t->checkpointStep.empty())
	{
		return M3D_GPU_ERR_ARGUMENT;
	}
	const int32_t n = t->nBodies;
	const size_t nn = (size_t)n;
	std::vector<BodyConst<float>> bcf(nn);
	std::vector<float> muf(nn), ef(nn);
	std::vector<m3d_diff::TapeShape> shapes(nn);
	cudaMemcpy(bcf.data(), t->bodyConst.ptr, sizeof(BodyConst<float>) * nn, cudaMemcpyDeviceToHost);
	cudaMemcpy(muf.data(), t->muBody.ptr, sizeof(float) * nn, cudaMemcpyDeviceToHost);
	cudaMemcpy(ef.data(), t->eBody.ptr, sizeof(float) * nn, cudaMemcpyDeviceToHost);
	cudaMemcpy(shapes.data(), t->shapes.ptr, sizeof(m3d_diff::TapeShape) * nn, cudaMemcpyDeviceToHost);
	std::vector<BodyConst<double>> bc(nn);
	std::vector<double> mu(nn), e(nn);
	for (size_t i = 0; i < nn; ++i)
	{
		bc[i].invMass = bcf[i].invMass;
		bc[i].il = bcf[i].il;
		bc[i].gravityScale = bcf[i].gravityScale;
		bc[i].linearDamping = bcf[i].linearDamping;
		bc[i].angularDamping = bcf[i].angularDamping;
		bc[i].dynamic = bcf[i].dynamic;
		mu[i] = muf[i];
		e[i] = ef[i];
	}
	const std::vector<HostStep> hs = downloadSteps(t);
	std::vector<Body<float>> ckAll = download<Body<float>>(t->checkpoints, 0, t->checkpointStep.size() * nn);
	HostArena arena;
	Work<double> k;
	const Limits lim = tapeLimits(t);
	carveWork(k, n, lim, [&](size_t b) { return arena(b); });
	packBodies(k.adj, n, dPos, dRot, dVel, dAngVel);
	typedef m3d_diff::ContactBar<double> Bar;
	Bar zero;
	m3d_diff::contactBarZero(zero);
	std::vector<Bar> bars[2];
	bars[0].assign((size_t)lim.positions, zero);
	bars[1].assign((size_t)lim.positions, zero);
	int cur = 0;
	auto ctx = [&](int step, const TapeStep& st, const HostStep& h) {
		const TapeContact* prev = nullptr;
		if (step > 0 && t->steps[step - 1].contactsPerSubstep > 0)
		{
			const TapeStep& p = t->steps[step - 1];
			prev = hs[step - 1].contacts.data() + (size_t)(p.substeps - 1) * (size_t)p.contactsPerSubstep;
		}
		return makeCtx<double>(k, bc.data(), mu.data(), e.data(), st, h.islands.data(), h.bodies.data(),
							   h.contacts.data(), n, bars[cur].data(), shapes.data(), prev,
							   h.prevPos.empty() ? nullptr : h.prevPos.data());
	};
	const int S = (int)t->steps.size();
	std::vector<Body<double>> states;
	for (int c = (int)t->checkpointStep.size() - 1; c >= 0; --c)
	{
		const int s0 = t->checkpointStep[c];
		const int s1 = c + 1 < (int)t->checkpointStep.size() ? t->checkpointStep[c + 1] : S;
		for (size_t i = 0; i < nn; ++i)
		{
			const Body<float>& b = ckAll[(size_t)c * nn + i];
			k.cur[i].x = m3d_diff::v3<double>(b.x.x, b.x.y, b.x.z);
			k.cur[i].q = m3d_diff::q4<double>(b.q.x, b.q.y, b.q.z, b.q.w);
			k.cur[i].v = m3d_diff::v3<double>(b.v.x, b.v.y, b.v.z);
			k.cur[i].w = m3d_diff::v3<double>(b.w.x, b.w.y, b.w.z);
		}
		states.assign((size_t)(s1 - s0) * nn, Body<double>());
		for (int step = s0; step < s1; ++step)
		{
			const TapeStep& st = t->steps[step];
			std::copy(k.cur, k.cur + nn, states.begin() + (ptrdiff_t)((size_t)(step - s0) * nn));
			IslandCtx<double> x = ctx(step, st, hs[step]);
			for (int q = 0; q < st.islands; ++q)
			{
				IslandCtx<double> y = x;
				y.island = hs[step].islands.data() + q;
				m3d_diff::islandStepForward(y);
			}
			for (uint32_t i : hs[step].sleeps)
			{
				k.cur[i].v = m3d_diff::vzero<double>();
				k.cur[i].w = m3d_diff::vzero<double>();
			}
		}
		for (int step = s1 - 1; step >= s0; --step)
		{
			const TapeStep& st = t->steps[step];
			for (uint32_t i : hs[step].sleeps)
			{
				k.adj[i].v = m3d_diff::vzero<double>();
				k.adj[i].w = m3d_diff::vzero<double>();
			}
			if (st.islands > 0)
			{
				const size_t off = (size_t)(step - s0) * nn;
				std::copy(states.begin() + (ptrdiff_t)off, states.begin() + (ptrdiff_t)(off + nn), k.cur);
				IslandCtx<double> x = ctx(step, st, hs[step]);
				for (int q = 0; q < st.islands; ++q)
				{
					IslandCtx<double> y = x;
					y.island = hs[step].islands.data() + q;
					m3d_diff::islandStepBackward(y);
				}
			}
			if (step > 0)
			{
				const TapeStep& pst = t->steps[step - 1];
				std::fill(bars[1 - cur].begin(), bars[1 - cur].begin() + pst.contactsPerSubstep, zero);
				for (int32_t p = 0; p < st.contactsPerSubstep && pst.contactsPerSubstep > 0; ++p)
				{
					if (hs[step].prevPos[p] >= 0)
					{
						bars[1 - cur][hs[step].prevPos[p]] = bars[cur][p];
					}
				}
				cur = 1 - cur;
			}
		}
	}
	const int32_t m = n < capacity ? n : capacity;
	unpackBodies(k.adj, m, gPos, gRot, gVel, gAngVel);
	for (int32_t i = 0; i < m; ++i)
	{
		if (gMass != nullptr)
		{
			gMass[i] = massGrad<double>(bcf[i], k.imBar[i], k.ilBar[i]);
		}
		if (gFriction != nullptr)
		{
			gFriction[i] = k.muBar[i];
		}
		if (gRestitution != nullptr)
		{
			gRestitution[i] = k.eBar[i];
		}
	}
	return M3D_GPU_OK;
}

// ---- regenerating replay (verification) ---------------------------------------------
//
// The recorded steps run again on the host from the first checkpoint, using
// only the tape's discrete record (islands, contact set, solve order, which
// contacts were regenerated when, sleeps) and regenerating every manifold at
// its recorded generation events from the current poses, with anchor
// inheritance and re-seating done live.  In float it must reproduce the
// engine bit for bit (then the tape captures every dependence of the step on
// the states); in double it is the smooth function whose derivative the
// adjoint computes, for central differences.

namespace
{
// perturbations (each may be null): initial linear and angular velocities
// (3 per body), masses, friction and restitution coefficients (1 per body)
struct Perturbation
{
	const double *dVel, *dAngVel, *dMass, *dFriction, *dRestitution;
};

template <typename T>
int32_t regenerateHost(DiffTape* t, const Perturbation& d, std::vector<Body<T>>& out)
{
	const int32_t n = t->nBodies;
	const size_t nn = (size_t)n;
	std::vector<BodyConst<float>> bcf(nn);
	std::vector<float> muf(nn), ef(nn);
	std::vector<m3d_diff::TapeShape> shapes(nn);
	cudaMemcpy(bcf.data(), t->bodyConst.ptr, sizeof(BodyConst<float>) * nn, cudaMemcpyDeviceToHost);
	cudaMemcpy(muf.data(), t->muBody.ptr, sizeof(float) * nn, cudaMemcpyDeviceToHost);
	cudaMemcpy(ef.data(), t->eBody.ptr, sizeof(float) * nn, cudaMemcpyDeviceToHost);
	cudaMemcpy(shapes.data(), t->shapes.ptr, sizeof(m3d_diff::TapeShape) * nn, cudaMemcpyDeviceToHost);
	std::vector<BodyConst<T>> bc(nn);
	std::vector<T> mu(nn), e(nn);
	for (size_t i = 0; i < nn; ++i)
	{
		bc[i].invMass = T(bcf[i].invMass);
		bc[i].il = T(bcf[i].il);
		bc[i].gravityScale = T(bcf[i].gravityScale);
		bc[i].linearDamping = T(bcf[i].linearDamping);
		bc[i].angularDamping = T(bcf[i].angularDamping);
		bc[i].dynamic = bcf[i].dynamic;
		mu[i] = T(muf[i]);
		e[i] = T(ef[i]);
		if (d.dMass != nullptr && bcf[i].dynamic && bcf[i].invMass > 0.0f)
		{
			// inertia scales with mass at fixed shape
			const double m = 1.0 / (double)bcf[i].invMass + d.dMass[i];
			const double im = 1.0 / m;
			bc[i].invMass = T(im);
			bc[i].il = T((double)bcf[i].il * im / (double)bcf[i].invMass);
		}
		if (d.dFriction != nullptr)
		{
			mu[i] = T((double)muf[i] + d.dFriction[i]);
		}
		if (d.dRestitution != nullptr)
		{
			e[i] = T((double)ef[i] + d.dRestitution[i]);
		}
	}
	const bool mixAgain = d.dFriction != nullptr || d.dRestitution != nullptr;
	const std::vector<HostStep> hs = downloadSteps(t);
	std::vector<Body<float>> ck = download<Body<float>>(t->checkpoints, 0, nn);
	std::vector<std::vector<T>> owned;
	auto alloc = [&](size_t bytes) {
		owned.emplace_back((bytes + sizeof(T) - 1) / sizeof(T), T(0));
		return (void*)owned.back().data();
	};
	Work<T> k;
	const Limits lim = tapeLimits(t);
	carveWork(k, n, lim, alloc);
	for (size_t i = 0; i < nn; ++i)
	{
		k.cur[i].x = m3d_diff::v3<T>(T(ck[i].x.x), T(ck[i].x.y), T(ck[i].x.z));
		k.cur[i].q = m3d_diff::q4<T>(T(ck[i].q.x), T(ck[i].q.y), T(ck[i].q.z), T(ck[i].q.w));
		k.cur[i].v = m3d_diff::v3<T>(T(ck[i].v.x), T(ck[i].v.y), T(ck[i].v.z));
		k.cur[i].w = m3d_diff::v3<T>(T(ck[i].w.x), T(ck[i].w.y), T(ck[i].w.z));
		if (d.dVel != nullptr)
		{
			k.cur[i].v = m3d_diff::v3<T>(T((double)ck[i].v.x + d.dVel[3 * i]), T((double)ck[i].v.y + d.dVel[3 * i + 1]),
										 T((double)ck[i].v.z + d.dVel[3 * i + 2]));
		}
		if (d.dAngVel != nullptr)
		{
			k.cur[i].w =
				m3d_diff::v3<T>(T((double)ck[i].w.x + d.dAngVel[3 * i]), T((double)ck[i].w.y + d.dAngVel[3 * i + 1]),
								T((double)ck[i].w.z + d.dAngVel[3 * i + 2]));
		}
	}
	std::vector<m3d_diff::Contact<T>> live[2];
	std::vector<uint32_t> liveIds[2];
	for (int b = 0; b < 2; ++b)
	{
		live[b].resize((size_t)lim.positions);
		liveIds[b].assign(4 * (size_t)lim.positions, 0u);
	}
	int L = 0;
	for (size_t step = 0; step < t->steps.size(); ++step)
	{
		const TapeStep& st = t->steps[step];
		const HostStep& h = hs[step];
		IslandCtx<T> x = makeCtx<T>(k, bc.data(), mu.data(), e.data(), st, h.islands.data(), h.bodies.data(),
									h.contacts.data(), n, nullptr, shapes.data());
		x.live = live[L].data();
		x.liveIds = liveIds[L].data();
		for (int32_t p = 0; p < st.contactsPerSubstep; ++p)
		{
			const TapeContact& rec = h.contacts[p];
			const int32_t prev = step > 0 && !h.prevPos.empty() ? h.prevPos[p] : -1;
			if (prev >= 0)
			{
				live[L][p] = live[1 - L][prev];
				for (int q = 0; q < 4; ++q)
				{
					liveIds[L][4 * p + q] = liveIds[1 - L][4 * prev + q];
				}
			}
			else
			{
				// the manifold the step began with is not on the tape: the
				// recorded one, or none when this step's narrowphase made it
				// (a contact that starts touching)
				live[L][p] = m3d_diff::loadContact<T>(rec);
				for (int q = 0; q < 4; ++q)
				{
					liveIds[L][4 * p + q] = rec.id[q];
				}
				if (step > 0 && (rec.gen & m3d_diff::kTapeGenNarrow))
				{
					live[L][p].pointCount = 0;
				}
			}
			// materials and shapes are the contact's own
			const m3d_diff::Contact<T> fromTape = m3d_diff::loadContact<T>(rec);
			live[L][p].a = fromTape.a;
			live[L][p].b = fromTape.b;
			live[L][p].curved = fromTape.curved;
			live[L][p].shapeA = fromTape.shapeA;
			live[L][p].shapeB = fromTape.shapeB;
			live[L][p].radiusA = fromTape.radiusA;
			live[L][p].radiusB = fromTape.radiusB;
			live[L][p].mu = fromTape.mu;
			live[L][p].e = fromTape.e;
			live[L][p].rolling = fromTape.rolling;
			if (mixAgain)
			{
				// contact materials from the perturbed body values, mixed as
				// contact creation mixes them
				live[L][p].mu = m3d_diff::dsqrt(mu[rec.a] * mu[rec.b]);
				live[L][p].e = e[rec.a] > e[rec.b] ? e[rec.a] : e[rec.b];
			}
			if (step > 0 && (rec.gen & m3d_diff::kTapeGenNarrow))
			{
				const Body<T>& A = k.cur[rec.a];
				const Body<T>& B = k.cur[rec.b];
				m3d_diff::regenerateLive(x, rec, p, A.x, A.q, B.x, B.q,
										 T(m3d_diff::kGenSpeculativeBase) + x.dt * m3d_diff::len(m3d_diff::sub(A.v, B.v)));
			}
		}
		for (int q = 0; q < st.islands; ++q)
		{
			IslandCtx<T> y = x;
			y.island = h.islands.data() + q;
			m3d_diff::islandStepForward(y);
		}
		for (uint32_t i : h.sleeps)
		{
			k.cur[i].v = m3d_diff::vzero<T>();
			k.cur[i].w = m3d_diff::vzero<T>();
		}
		L = 1 - L;
	}
	out.assign(k.cur, k.cur + nn);
	return M3D_GPU_OK;
}
} // namespace

int32_t tapeRegenerateHost(DiffTape* t, int doublePrecision, const double* dVel, const double* dAngVel,
						   const double* dMass, const double* dFriction, const double* dRestitution, double* pos,
						   double* rot, double* vel, double* angVel, int32_t capacity)
{
	if (t->steps.empty() || t->checkpointStep.empty())
	{
		return M3D_GPU_ERR_ARGUMENT;
	}
	const int32_t m = t->nBodies < capacity ? t->nBodies : capacity;
	const Perturbation d = { dVel, dAngVel, dMass, dFriction, dRestitution };
	if (doublePrecision)
	{
		std::vector<Body<double>> out;
		int32_t rc = regenerateHost<double>(t, d, out);
		unpackBodies(out.data(), m, pos, rot, vel, angVel);
		return rc;
	}
	std::vector<Body<float>> out;
	int32_t rc = regenerateHost<float>(t, d, out);
	unpackBodies(out.data(), m, pos, rot, vel, angVel);
	return rc;
}

} // namespace m3g

// Island solve of one step: all substeps of every awake island.
//
//  - free islands (one body, no contacts, no joints): integrate and
//    reconstruct per substep, one thread per body;
//  - small islands (< 300 contacts): the reference's serial Gauss-Seidel in
//    ascending contact order (src/xpbd.cpp:898-974), one thread per island
//    for the smallest (up to 8 contacts, no joints), one warp otherwise;
//  - giant islands (k_giant.cu) take the whole GPU;
//  - big islands (>= 300 contacts): the reference's graph-coloured solve
//    (src/xpbd.cpp:1167-1369), one CTA per island: greedy first-fit colouring
//    in contact order, colour buckets solved in parallel (bodies in a bucket
//    are disjoint), the overflow bucket and the joints serially, with
//    __syncthreads() where the reference joins its fork-join stages.
// Islands are disjoint in their dynamic bodies, so all islands run at once.
#include "m3d_dev.cuh"
#include "m3d_diff.h"
#include "m3d_solve.cuh"

namespace m3g
{


__global__ void kSolveFree(BodySoA B, const IslandRec* islands, int32_t ni, const uint32_t* islandsDev,
						   const uint32_t* bodyVals, SolveParams P)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= ni || k >= (int)*islandsDev)
	{
		return;
	}
	const IslandRec r = islands[k];
	if (r.kind != 0)
	{
		return;
	}
	for (int b = 0; b < r.bodyCount; ++b)
	{
		int i = (int)bodyVals[r.bodyStart + b];
		for (int sub = 0; sub < P.substeps; ++sub)
		{
			integrateBody(B, i, P.h, P.gravity);
			reconstructBody(B, i, P.invH);
		}
	}
}

// One warp per small island.  The per-element stages of a substep whose
// elements are independent - integration and velocity reconstruction of each
// body, preparation of each contact (which reads only body state and writes
// only its own contact) - run across the lanes.
//
// The Gauss-Seidel sweeps follow the reference's ascending contact order
// exactly, but not one contact at a time: a contact reads and writes only its
// own records and the two bodies it joins, and only bodies with non-zero
// inverse mass are ever written, so two contacts that share no island body
// commute.  Each contact gets the level 1 + max(level of the previous contact
// on each of its island bodies); a sweep runs level by level, the contacts of
// one level in parallel.  Every contact still sees each body exactly as the
// serial sweep leaves it.  Islands with joints, or larger than the shared
// tables, sweep serially on lane 0.  __syncwarp() orders the global-memory
// writes of one stage or level before the reads of the next.
// Differentiation tape: the manifold of a contact right after its
// preparation in one substep, with the point ids and how the manifold came to
// be (what the adjoint holds as the record of the forward).
static_assert(kPrepRegenerated == m3d_diff::kTapeGenPrepare && kPrepHeld == m3d_diff::kTapeGenHeld,
			  "tape generation flags follow the preparation flags");

__device__ void writeTapeContact(m3d_diff::TapeContact& t, const BodySoA& B, const ContactSoA& C, int c, int gen)
{
	const int2 ab = C.bodies[c];
	const BodyCold& ca = B.cold[ab.x];
	const BodyCold& cb = B.cold[ab.y];
	t.gen = gen;
	t.a = ab.x;
	t.b = ab.y;
	t.pointCount = C.pointCount[c];
	t.curved = (C.flags[c] & kCFCurved) != 0 ? 1 : 0;
	t.shapeA = (int32_t)ca.shape.type;
	t.shapeB = (int32_t)cb.shape.type;
	t.radiusA = ca.shape.radius;
	t.radiusB = cb.shape.radius;
	const float4 n = C.normal[c];
	t.n[0] = n.x;
	t.n[1] = n.y;
	t.n[2] = n.z;
	t.mu = n.w;
	const float2 mat = C.mat[c];
	t.e = mat.x;
	t.rolling = mat.y;
	for (int s = 0; s < 4; ++s)
	{
		const size_t k = pidx(C, c, s);
		const float4 la = C.pAnchorA[k], lb = C.pAnchorB[k], fa = C.pFricA[k], fb = C.pFricB[k], sl = C.pSlip[k];
		t.la[s][0] = la.x, t.la[s][1] = la.y, t.la[s][2] = la.z;
		t.lb[s][0] = lb.x, t.lb[s][1] = lb.y, t.lb[s][2] = lb.z;
		t.fa[s][0] = fa.x, t.fa[s][1] = fa.y, t.fa[s][2] = fa.z;
		t.fb[s][0] = fb.x, t.fb[s][1] = fb.y, t.fb[s][2] = fb.z;
		t.slip[s][0] = sl.x, t.slip[s][1] = sl.y, t.slip[s][2] = sl.z;
		t.off[s] = sl.w;
		t.id[s] = __float_as_uint(lb.w);
	}
}

constexpr int kSerialWarpsPerBlock = 8;
constexpr int kLevelTable = 320; // contacts and bodies per island for the level schedule
constexpr uint32_t kNotIsland = 0xFFFFu;

// Level schedules of one island (see kSolveSerial).  Positions index the
// island's contacts; for islands with joints, the position sweeps run over
// the joints followed by the contacts (the reference projects the joints
// first in each iteration) and the velocity pass over the contacts followed
// by the joints (it runs the joint motors after the contacts).
struct LevelTables
{
	uint32_t contact[kLevelTable];  // contact index per island position
	uint32_t ends[kLevelTable];     // island-local body of each end (kNotIsland: static / kinematic / other)
	uint16_t level[kLevelTable];    // 1-based level per contact (friction sweep; every sweep without joints)
	uint16_t last[kLevelTable];     // per island body: level of its latest element
	uint16_t levelPos[kLevelTable]; // joints then contacts: level in the position sweeps
	uint16_t levelVel[kLevelTable]; // contacts then joints: level in the velocity pass
};

// lane 0: levels of a sequence of elements given by their two island-local
// ends; each element one level above the latest earlier element on either end
__device__ __forceinline__ uint16_t levelOf(LevelTables& T, uint32_t la, uint32_t lb)
{
	uint16_t l = 0;
	if (la != kNotIsland)
	{
		l = T.last[la];
	}
	if (lb != kNotIsland && T.last[lb] > l)
	{
		l = T.last[lb];
	}
	++l;
	if (la != kNotIsland)
	{
		T.last[la] = l;
	}
	if (lb != kNotIsland)
	{
		T.last[lb] = l;
	}
	return l;
}

enum SweepOp
{
	kSweepNormals,
	kSweepFriction,
	kSweepVelocity
};

__device__ __forceinline__ void sweepContact(SweepOp op, const BodySoA& B, const ContactSoA& C, int c,
											 const SolveParams& P)
{
	if (op == kSweepNormals)
	{
		solveContactNormals(B, C, c, P.maxCorrection);
	}
	else if (op == kSweepFriction)
	{
		applyContactFriction(B, C, c);
	}
	else
	{
		solveContactVelocity(B, C, c, P.h, P.gravityLen);
	}
}

// one sweep over the joints and contacts of an island with joints, level by
// level (position: joints then contacts; velocity: contacts then joints)
__device__ __forceinline__ void sweepJointedIsland(bool position, const BodySoA& B, const ContactSoA& C, JointRec* J,
												   const IslandRec& r, const uint32_t* joints, const LevelTables& T,
												   int levels, int lane, const SolveParams& P)
{
	const int nj = r.jointCount, nc = r.contactCount;
	const uint16_t* lev = position ? T.levelPos : T.levelVel;
	for (int L = 1; L <= levels; ++L)
	{
		for (int q = lane; q < nj + nc; q += 32)
		{
			if (lev[q] != L)
			{
				continue;
			}
			const bool isJoint = position ? q < nj : q >= nc;
			if (isJoint)
			{
				const int j = (int)joints[position ? q : q - nc];
				if (position)
				{
					jointPosition(B, J, j, P.h);
				}
				else
				{
					jointVelocity(B, J, j, P.h);
				}
			}
			else
			{
				const int c = (int)T.contact[position ? q - nj : q];
				if (position)
				{
					solveContactNormals(B, C, c, P.maxCorrection);
				}
				else
				{
					solveContactVelocity(B, C, c, P.h, P.gravityLen);
				}
			}
		}
		__syncwarp();
	}
}

// one Gauss-Seidel sweep over the island's contacts in reference order
__device__ __forceinline__ void sweepIsland(SweepOp op, const BodySoA& B, const ContactSoA& C, const IslandRec& r,
											const uint32_t* contacts, const LevelTables& T, int levels, int lane,
											const SolveParams& P)
{
	if (levels > 0)
	{
		for (int L = 1; L <= levels; ++L)
		{
			for (int p = lane; p < r.contactCount; p += 32)
			{
				if (T.level[p] == L)
				{
					sweepContact(op, B, C, (int)T.contact[p], P);
				}
			}
			__syncwarp();
		}
	}
	else
	{
		if (lane == 0)
		{
			for (int c = 0; c < r.contactCount; ++c)
			{
				sweepContact(op, B, C, (int)contacts[c], P);
			}
		}
		__syncwarp();
	}
}

// kTape: the instance used while a differentiation tape records (the plain
// instance carries none of the recording code)
template <bool kTape>
__global__ void __launch_bounds__(32 * kSerialWarpsPerBlock)
	kSolveSerial(BodySoA B, ContactSoA C, JointRec* J, const IslandRec* islands, const int32_t* serialList,
				 const uint32_t* serialDev, const uint32_t* bodyVals, const uint32_t* contactVals,
				 const uint32_t* jointVals, uint32_t* localIndex, SolveParams P, m3d_diff::TapeContact* tape,
				 const uint32_t* tapeStride, const uint8_t* narrowGen)
{
	M3G_KERNEL_BEGIN();
	__shared__ LevelTables tables[kSerialWarpsPerBlock];
	const int lane = threadIdx.x & 31;
	LevelTables& T = tables[threadIdx.x >> 5];
	const int warps = gridDim.x * kSerialWarpsPerBlock;
	const int count = (int)*serialDev;
	for (int si = blockIdx.x * kSerialWarpsPerBlock + (threadIdx.x >> 5); si < count; si += warps)
	{
		const IslandRec r = islands[serialList[si]];
		const uint32_t* bodies = bodyVals + r.bodyStart;
		const uint32_t* contacts = contactVals + r.contactStart;
		const uint32_t* joints = jointVals + r.jointStart;

		// level schedules of the island's contacts and joints (fixed for the
		// whole step)
		int levels = 0, levelsPos = 0, levelsVel = 0;
		const int nj = r.jointCount, nc = r.contactCount;
		if (nc + nj <= kLevelTable && r.bodyCount <= kLevelTable)
		{
			for (int b = lane; b < r.bodyCount; b += 32)
			{
				localIndex[bodies[b]] = (uint32_t)b;
				T.last[b] = 0;
			}
			__syncwarp();
			for (int p = lane; p < nc; p += 32)
			{
				const uint32_t c = contacts[p];
				const int2 ab = C.bodies[c];
				uint32_t la = localIndex[ab.x], lb = localIndex[ab.y];
				la = la < (uint32_t)r.bodyCount && bodies[la] == (uint32_t)ab.x ? la : kNotIsland;
				lb = lb < (uint32_t)r.bodyCount && bodies[lb] == (uint32_t)ab.y ? lb : kNotIsland;
				T.contact[p] = c;
				T.ends[p] = la | (lb << 16);
			}
			__syncwarp();
			if (lane == 0)
			{
				for (int p = 0; p < nc; ++p)
				{
					T.level[p] = levelOf(T, T.ends[p] & 0xFFFFu, T.ends[p] >> 16);
					levels = T.level[p] > levels ? T.level[p] : levels;
				}
				if (nj > 0)
				{
					// a joint's island-local ends (its static or kinematic end,
					// never written, does not order anything)
					auto jointEnds = [&](int q, uint32_t& la, uint32_t& lb) {
						const JointRec& jr = J[joints[q]];
						la = localIndex[jr.bodyA];
						lb = localIndex[jr.bodyB];
						la = la < (uint32_t)r.bodyCount && bodies[la] == (uint32_t)jr.bodyA ? la : kNotIsland;
						lb = lb < (uint32_t)r.bodyCount && bodies[lb] == (uint32_t)jr.bodyB ? lb : kNotIsland;
					};
					for (int b = 0; b < r.bodyCount; ++b)
					{
						T.last[b] = 0;
					}
					for (int q = 0; q < nj + nc; ++q)
					{
						uint32_t la, lb;
						if (q < nj)
						{
							jointEnds(q, la, lb);
						}
						else
						{
							la = T.ends[q - nj] & 0xFFFFu;
							lb = T.ends[q - nj] >> 16;
						}
						T.levelPos[q] = levelOf(T, la, lb);
						levelsPos = T.levelPos[q] > levelsPos ? T.levelPos[q] : levelsPos;
					}
					for (int b = 0; b < r.bodyCount; ++b)
					{
						T.last[b] = 0;
					}
					for (int q = 0; q < nj + nc; ++q)
					{
						uint32_t la, lb;
						if (q < nc)
						{
							la = T.ends[q] & 0xFFFFu;
							lb = T.ends[q] >> 16;
						}
						else
						{
							jointEnds(q - nc, la, lb);
						}
						T.levelVel[q] = levelOf(T, la, lb);
						levelsVel = T.levelVel[q] > levelsVel ? T.levelVel[q] : levelsVel;
					}
				}
			}
			levels = __shfl_sync(0xffffffffu, levels, 0);
			levelsPos = __shfl_sync(0xffffffffu, levelsPos, 0);
			levelsVel = __shfl_sync(0xffffffffu, levelsVel, 0);
			__syncwarp();
		}
		// islands with joints but too large for the tables stay serial on lane 0
		const bool jointsLevelled = nj > 0 && levelsPos > 0;
		if (nj > 0 && !jointsLevelled)
		{
			levels = 0;
		}

		if (r.jointCount > 0)
		{
			for (int b = lane; b < r.bodyCount; b += 32)
			{
				refreshInvInertia(B, (int)bodies[b]);
			}
			__syncwarp();
			// each joint's preparation reads the bodies and writes only its own
			// record: any order gives the same records
			for (int j = lane; j < r.jointCount; j += 32)
			{
				jointPrepare(B, J, (int)joints[j]);
			}
			__syncwarp();
		}
		for (int sub = 0; sub < P.substeps; ++sub)
		{
			for (int b = lane; b < r.bodyCount; b += 32)
			{
				integrateBody(B, (int)bodies[b], P.h, P.gravity);
			}
			__syncwarp();
			for (int c = lane; c < r.contactCount; c += 32)
			{
				const int what = prepareContact(B, C, (int)contacts[c], P.h);
				if (kTape && tape != nullptr)
				{
					int gen = what;
					if (sub == 0 && narrowGen[contacts[c]] == kPrepRegenerated)
					{
						gen |= m3d_diff::kTapeGenNarrow;
					}
					writeTapeContact(tape[(size_t)sub * *tapeStride + r.contactStart + c], B, C, (int)contacts[c], gen);
				}
			}
			__syncwarp();
			if (jointsLevelled)
			{
				for (int j = lane; j < r.jointCount; j += 32)
				{
					jointReset(J, (int)joints[j]);
				}
				__syncwarp();
				for (int it = 0; it < P.iterations; ++it)
				{
					sweepJointedIsland(true, B, C, J, r, joints, T, levelsPos, lane, P);
				}
			}
			else if (r.jointCount > 0)
			{
				// joints interleave with the contact sweeps: serial on lane 0
				if (lane == 0)
				{
					for (int j = 0; j < r.jointCount; ++j)
					{
						jointReset(J, (int)joints[j]);
					}
					for (int it = 0; it < P.iterations; ++it)
					{
						for (int j = 0; j < r.jointCount; ++j)
						{
							jointPosition(B, J, (int)joints[j], P.h);
						}
						for (int c = 0; c < r.contactCount; ++c)
						{
							solveContactNormals(B, C, (int)contacts[c], P.maxCorrection);
						}
					}
				}
				__syncwarp();
			}
			else
			{
				for (int it = 0; it < P.iterations; ++it)
				{
					sweepIsland(kSweepNormals, B, C, r, contacts, T, levels, lane, P);
				}
			}
			sweepIsland(kSweepFriction, B, C, r, contacts, T, levels, lane, P);
			for (int b = lane; b < r.bodyCount; b += 32)
			{
				reconstructBody(B, (int)bodies[b], P.invH);
			}
			__syncwarp();
			if (jointsLevelled)
			{
				sweepJointedIsland(false, B, C, J, r, joints, T, levelsVel, lane, P);
			}
			else
			{
				sweepIsland(kSweepVelocity, B, C, r, contacts, T, levels, lane, P);
				if (lane == 0)
				{
					for (int j = 0; j < r.jointCount; ++j)
					{
						jointVelocity(B, J, (int)joints[j], P.h);
					}
				}
				__syncwarp();
			}
		}
	}
}

// Small serial islands without joints, one thread each: the whole substep
// loop in the reference's order (src/xpbd.cpp:898-974), 32 islands per warp.
template <bool kTape>
__global__ void __launch_bounds__(128)
	kSolveTiny(BodySoA B, ContactSoA C, const IslandRec* islands, const int32_t* tinyList, const uint32_t* tinyDev,
			   const uint32_t* bodyVals, const uint32_t* contactVals, SolveParams P, m3d_diff::TapeContact* tape,
			   const uint32_t* tapeStride, const uint8_t* narrowGen)
{
	M3G_KERNEL_BEGIN();
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= (int)*tinyDev)
	{
		return;
	}
	const IslandRec r = islands[tinyList[k]];
	const uint32_t* bodies = bodyVals + r.bodyStart;
	const uint32_t* contacts = contactVals + r.contactStart;
	for (int sub = 0; sub < P.substeps; ++sub)
	{
		for (int b = 0; b < r.bodyCount; ++b)
		{
			integrateBody(B, (int)bodies[b], P.h, P.gravity);
		}
		for (int c = 0; c < r.contactCount; ++c)
		{
			const int what = prepareContact(B, C, (int)contacts[c], P.h);
			if (kTape && tape != nullptr)
			{
				int gen = what;
				if (sub == 0 && narrowGen[contacts[c]] == kPrepRegenerated)
				{
					gen |= m3d_diff::kTapeGenNarrow;
				}
				writeTapeContact(tape[(size_t)sub * *tapeStride + r.contactStart + c], B, C, (int)contacts[c], gen);
			}
		}
		for (int it = 0; it < P.iterations; ++it)
		{
			for (int c = 0; c < r.contactCount; ++c)
			{
				solveContactNormals(B, C, (int)contacts[c], P.maxCorrection);
			}
		}
		for (int c = 0; c < r.contactCount; ++c)
		{
			applyContactFriction(B, C, (int)contacts[c]);
		}
		for (int b = 0; b < r.bodyCount; ++b)
		{
			reconstructBody(B, (int)bodies[b], P.invH);
		}
		for (int c = 0; c < r.contactCount; ++c)
		{
			solveContactVelocity(B, C, (int)contacts[c], P.h, P.gravityLen);
		}
	}
}

constexpr int kColorThreads = 256;

__device__ void colorIsland(BodySoA B, ContactSoA C, JointRec* J, const IslandRec r, const uint32_t* bodyVals,
							const uint32_t* contactVals, const uint32_t* jointVals, uint32_t* colorMask,
							int32_t* colorOrder, int32_t* packetMax, int32_t* contactColor, SolveParams P,
							int32_t* bucketStart, int32_t* colorCountPtr)
{
	int32_t& colorCount = *colorCountPtr;
	const int tid = threadIdx.x, nt = blockDim.x;
	const uint32_t* bodies = bodyVals + r.bodyStart;
	const uint32_t* contacts = contactVals + r.contactStart;
	const uint32_t* joints = jointVals + r.jointStart;
	int32_t* order = colorOrder + r.contactStart;
	int32_t* pmax = packetMax + r.contactStart;

	// ---- greedy first-fit colouring in contact order (src/xpbd.cpp:1179-1235)
	for (int b = tid; b < r.bodyCount; b += nt)
	{
		colorMask[bodies[b]] = 0;
	}
	__syncthreads();
	if (tid == 0)
	{
		int32_t counts[kMaxGraphColors + 1];
		for (int c = 0; c <= kMaxGraphColors; ++c)
		{
			counts[c] = 0;
		}
		int32_t cc = 0;
		// pass 1: colours (stored temporarily in `order`)
		for (int p = 0; p < r.contactCount; ++p)
		{
			int ci = (int)contacts[p];
			int2 ab = C.bodies[ci];
			bool dynA = B.massInv[ab.x].x > 0.0f;
			bool dynB = B.massInv[ab.y].x > 0.0f;
			uint32_t used = 0;
			if (dynA)
			{
				used |= colorMask[ab.x];
			}
			if (dynB)
			{
				used |= colorMask[ab.y];
			}
			uint32_t freeBits = ~used;
			int color = freeBits != 0 ? __ffs((int)freeBits) - 1 : kMaxGraphColors;
			if (color >= kMaxGraphColors)
			{
				color = kMaxGraphColors;
			}
			else
			{
				uint32_t bit = 1u << color;
				if (dynA)
				{
					colorMask[ab.x] |= bit;
				}
				if (dynB)
				{
					colorMask[ab.y] |= bit;
				}
				cc = color + 1 > cc ? color + 1 : cc;
			}
			order[p] = color;
			contactColor[ci] = color;
			++counts[color];
		}
		int32_t run = 0;
		for (int c = 0; c <= kMaxGraphColors; ++c)
		{
			bucketStart[c] = run;
			run += counts[c];
		}
		bucketStart[kMaxGraphColors + 1] = run;
		colorCount = cc;
		// pass 2: regroup by colour, keeping contact order inside each bucket
		int32_t cursor[kMaxGraphColors + 1];
		for (int c = 0; c <= kMaxGraphColors; ++c)
		{
			cursor[c] = bucketStart[c];
		}
		for (int p = 0; p < r.contactCount; ++p)
		{
			int color = contactColor[contacts[p]];
			pmax[cursor[color]++] = (int32_t)contacts[p];
		}
		for (int p = 0; p < r.contactCount; ++p)
		{
			order[p] = pmax[p];
		}
	}
	__syncthreads();
	const int ncol = colorCount;

	if (r.jointCount > 0)
	{
		for (int b = tid; b < r.bodyCount; b += nt)
		{
			refreshInvInertia(B, (int)bodies[b]);
		}
		__syncthreads();
		if (tid == 0)
		{
			for (int j = 0; j < r.jointCount; ++j)
			{
				jointPrepare(B, J, (int)joints[j]);
			}
		}
		__syncthreads();
	}

	const int colored = bucketStart[kMaxGraphColors];
	const int overflowStart = colored, overflowEnd = bucketStart[kMaxGraphColors + 1];
	for (int sub = 0; sub < P.substeps; ++sub)
	{
		for (int b = tid; b < r.bodyCount; b += nt)
		{
			integrateBody(B, (int)bodies[b], P.h, P.gravity);
		}
		__syncthreads();
		for (int c = tid; c < r.contactCount; c += nt)
		{
			prepareContact(B, C, (int)contacts[c], P.h);
		}
		if (tid == 0)
		{
			for (int j = 0; j < r.jointCount; ++j)
			{
				jointReset(J, (int)joints[j]);
			}
		}
		__syncthreads();
		// packets of 8 consecutive bucket entries share the largest point count
		for (int q = tid; q < colored; q += nt)
		{
			int color = 0;
			while (q >= bucketStart[color + 1])
			{
				++color;
			}
			int bs = bucketStart[color], be = bucketStart[color + 1];
			int p0 = bs + ((q - bs) & ~7);
			int p1 = p0 + 8 < be ? p0 + 8 : be;
			int m = 0;
			for (int p = p0; p < p1; ++p)
			{
				int pc = C.pointCount[order[p]];
				m = pc > m ? pc : m;
			}
			pmax[q] = m;
		}
		__syncthreads();
		for (int it = 0; it < P.iterations; ++it)
		{
			if (tid == 0)
			{
				for (int j = 0; j < r.jointCount; ++j)
				{
					jointPosition(B, J, (int)joints[j], P.h);
				}
			}
			__syncthreads();
			for (int color = 0; color < ncol; ++color)
			{
				for (int q = bucketStart[color] + tid; q < bucketStart[color + 1]; q += nt)
				{
					solvePacketLane(B, C, order[q], pmax[q], P.maxCorrection);
				}
				__syncthreads();
			}
			if (tid == 0)
			{
				for (int q = overflowStart; q < overflowEnd; ++q)
				{
					solveContactNormals(B, C, order[q], P.maxCorrection);
				}
			}
			__syncthreads();
		}
		for (int color = 0; color < ncol; ++color)
		{
			for (int q = bucketStart[color] + tid; q < bucketStart[color + 1]; q += nt)
			{
				applyContactFriction(B, C, order[q]);
			}
			__syncthreads();
		}
		if (tid == 0)
		{
			for (int q = overflowStart; q < overflowEnd; ++q)
			{
				applyContactFriction(B, C, order[q]);
			}
		}
		__syncthreads();
		for (int b = tid; b < r.bodyCount; b += nt)
		{
			reconstructBody(B, (int)bodies[b], P.invH);
		}
		__syncthreads();
		for (int color = 0; color < ncol; ++color)
		{
			for (int q = bucketStart[color] + tid; q < bucketStart[color + 1]; q += nt)
			{
				solveContactVelocity(B, C, order[q], P.h, P.gravityLen);
			}
			__syncthreads();
		}
		if (tid == 0)
		{
			for (int q = overflowStart; q < overflowEnd; ++q)
			{
				solveContactVelocity(B, C, order[q], P.h, P.gravityLen);
			}
			for (int j = 0; j < r.jointCount; ++j)
			{
				jointVelocity(B, J, (int)joints[j], P.h);
			}
		}
		__syncthreads();
	}
}

__global__ void __launch_bounds__(kColorThreads)
	kSolveColored(BodySoA B, ContactSoA C, JointRec* J, const IslandRec* islands, const int32_t* coloredList,
				  const uint32_t* coloredDev, const uint32_t* bodyVals, const uint32_t* contactVals,
				  const uint32_t* jointVals, uint32_t* colorMask, int32_t* colorOrder, int32_t* packetMax,
				  int32_t* contactColor, SolveParams P)
{
	M3G_KERNEL_BEGIN();
	__shared__ int32_t bucketStart[kMaxGraphColors + 2];
	__shared__ int32_t colorCount;
	for (int ci = blockIdx.x; ci < (int)*coloredDev; ci += gridDim.x)
	{
		colorIsland(B, C, J, islands[coloredList[ci]], bodyVals, contactVals, jointVals, colorMask, colorOrder,
					packetMax, contactColor, P, bucketStart, &colorCount);
		__syncthreads();
	}
}

void launchSolve(DevWorld& w, float dt, int substeps, V3 gravity, int positionIterations)
{
	StepCounters* dc = devCounters(w);
	int32_t ni = w.islandMax; // upper bound; the exact island count is on the device
	if (ni <= 0)
	{
		return;
	}
	SolveParams P;
	P.h = dt / (float)substeps;
	P.invH = P.h > 0.0f ? 1.0f / P.h : 0.0f;
	P.maxCorrection = kMaxDepenetrationSpeed * P.h;
	P.gravity = gravity;
	P.gravityLen = len(gravity);
	P.substeps = substeps;
	P.iterations = positionIterations > 0 ? positionIterations : 2;
	cudaStream_t s = w.stream;
	const IslandRec* isl = w.islands.as<IslandRec>();
	M3G_LAUNCH(kSolveFree, blocksFor(ni, 128), 128, s, w.B, isl, ni, &dc->awakeIslands, w.bodyVals.as<uint32_t>(), P);
	// enough warps for every serial island of a rain or pile step to start at once
	int serialBlocks = (ni + kSerialWarpsPerBlock - 1) / kSerialWarpsPerBlock;
	serialBlocks = serialBlocks < 148 * 8 ? serialBlocks : 148 * 8;
	w.colorMask.ensure((size_t)(w.bodyCap + 1) * sizeof(uint32_t)); // also the serial islands' local body index
	if (w.lastSerialIslands > w.tinyModeIslands) // the island table listed tiny islands this step
	{
		if (w.tapeContacts != nullptr)
		{
			M3G_LAUNCH_AS("kSolveTiny", kSolveTiny<true>, blocksFor(ni, 128), 128, s, w.B, w.C, isl,
						  w.tinyList.as<int32_t>(), &dc->tinyIslands, w.bodyVals.as<uint32_t>(),
						  w.contactVals.as<uint32_t>(), P, w.tapeContacts, &dc->islandContacts, w.tapeGen.as<uint8_t>());
		}
		else
		{
			M3G_LAUNCH_AS("kSolveTiny", kSolveTiny<false>, blocksFor(ni, 128), 128, s, w.B, w.C, isl,
						  w.tinyList.as<int32_t>(), &dc->tinyIslands, w.bodyVals.as<uint32_t>(),
						  w.contactVals.as<uint32_t>(), P, w.tapeContacts, &dc->islandContacts, w.tapeGen.as<uint8_t>());
		}
	}
	if (w.tapeContacts != nullptr)
	{
		M3G_LAUNCH_AS("kSolveSerial", kSolveSerial<true>, serialBlocks, 32 * kSerialWarpsPerBlock, s, w.B, w.C,
					  w.joints.as<JointRec>(), isl, w.serialList.as<int32_t>(), &dc->warpIslands,
					  w.bodyVals.as<uint32_t>(), w.contactVals.as<uint32_t>(), w.jointVals.as<uint32_t>(),
					  w.colorMask.as<uint32_t>(), P, w.tapeContacts, &dc->islandContacts, w.tapeGen.as<uint8_t>());
	}
	else
	{
		M3G_LAUNCH_AS("kSolveSerial", kSolveSerial<false>, serialBlocks, 32 * kSerialWarpsPerBlock, s, w.B, w.C,
					  w.joints.as<JointRec>(), isl, w.serialList.as<int32_t>(), &dc->warpIslands,
					  w.bodyVals.as<uint32_t>(), w.contactVals.as<uint32_t>(), w.jointVals.as<uint32_t>(),
					  w.colorMask.as<uint32_t>(), P, w.tapeContacts, &dc->islandContacts, w.tapeGen.as<uint8_t>());
	}
	size_t nc = (size_t)w.contactMax + 1;
	w.colorOrder.ensure(nc * sizeof(int32_t));
	w.packetMax.ensure(nc * sizeof(int32_t));
	M3G_LAUNCH(kSolveColored, 2 * 148, kColorThreads, s, w.B, w.C, w.joints.as<JointRec>(), isl,
			   w.coloredList.as<int32_t>(), &dc->coloredIslands, w.bodyVals.as<uint32_t>(), w.contactVals.as<uint32_t>(),
			   w.jointVals.as<uint32_t>(), w.colorMask.as<uint32_t>(), w.colorOrder.as<int32_t>(),
			   w.packetMax.as<int32_t>(), w.contactColor.as<int32_t>(), P);
	launchSolveGiant(w, P);
}

} // namespace m3g

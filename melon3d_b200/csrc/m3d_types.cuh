// Device-resident world layout and engine constants.
//
// Bodies and contacts are structure-of-arrays in HBM.  Vector fields are
// float4 (w unused or carrying a scalar) so a warp reads them as coalesced
// 16-byte loads.  Manifold points are stored point-slot major
// (index = slot * contactCapacity + contact) so the threads of a warp that
// handle consecutive contacts read consecutive addresses for a given slot.
#pragma once

#include "m3d_math.cuh"

#include <cuda_runtime.h>
#include <stdint.h>

namespace m3g
{

// ---- tuning constants (reference src/m3d_internal.h:32-63) ----------------
constexpr float kLinearSlop = 0.005f;
constexpr float kSpeculativeBase = 4.0f * kLinearSlop;
constexpr float kMaxDepenetrationSpeed = 3.0f;
constexpr float kFrictionRelaxation = 0.5f;
constexpr float kAABBMargin = 0.1f;
constexpr float kTimeToSleep = 0.5f;
constexpr float kSleepLinearVelSq = 0.05f * 0.05f;
constexpr float kSleepAngularVelSq = 0.05f * 0.05f;
constexpr float kSleepEnergyThresh = kSleepLinearVelSq + kSleepAngularVelSq;
constexpr float kSleepEnergyAlpha = 0.25f;
constexpr float kSleepWakeFactor = 3.0f;
constexpr int32_t kOversizedCellSpan = 64;
constexpr int32_t kBigIslandContacts = 300;
constexpr int32_t kMaxGraphColors = 8;
// Serial islands up to kTinyIslandContacts contacts (no joints) take one
// thread each when the previous step had more than kTinyModeIslands serial
// islands (throughput-bound: 32 islands per warp); with fewer, every serial
// island takes a warp (latency-bound: no divergence between islands).
constexpr int32_t kTinyIslandContacts = 8;
constexpr uint32_t kTinyModeIslands = 16384;

// body sidecar bits (reference src/m3d_internal.h:271-274)
constexpr uint8_t kBFDynamic = 1;
constexpr uint8_t kBFAwake = 2;
constexpr uint8_t kBFInUse = 4;
constexpr uint8_t kBFKinematic = 8;

// persistent per-body state bits (device `state` array)
constexpr uint8_t kStInUse = 1;
constexpr uint8_t kStAwake = 2;
constexpr uint8_t kStEnableSleep = 4;
constexpr uint8_t kStSensor = 8;

// contact flag bits
constexpr uint8_t kCFTouching = 1;
constexpr uint8_t kCFSensor = 2;
constexpr uint8_t kCFTunnelGuard = 4;
constexpr uint8_t kCFCurved = 8;
constexpr uint8_t kCFHasCache = 16;

enum ShapeType : int32_t
{
	kSphere = 0,
	kCapsule = 1,
	kBox = 2
};
enum BodyType : int32_t
{
	kStatic = 0,
	kKinematic = 1,
	kDynamic = 2
};
enum JointKind : int32_t
{
	kJointDistance = 0,
	kJointBall = 1,
	kJointHinge = 2,
	kJointWeld = 3
};

struct Shape
{
	int32_t type;
	float radius;
	float halfHeight;
	V3 he;
};

// Per-body fields that are set at creation (or by rare setters) and read by
// the broadphase filters and collision routines.
struct BodyCold
{
	Shape shape;
	float friction;
	float restitution;
	float rollingResistance;
	float gravityScale;
	float linearDamping;
	float angularDamping;
	uint32_t categoryBits;
	uint32_t maskBits;
	int32_t groupIndex;
	int32_t type;
};

struct ManifoldPoint
{
	V3 localAnchorA;
	V3 localAnchorB;
	V3 frictionAnchorA;
	V3 frictionAnchorB;
	float separation;
	uint32_t id;
	float lambdaN;
	float lambdaT;
	float separationOffset;
	V3 slipDir;
};

struct Manifold
{
	V3 normal;
	int32_t pointCount;
	ManifoldPoint points[4];
};

// Joint record, identical on host and device (reference src/m3d_internal.h:313-349)
struct JointRec
{
	int32_t type;
	int32_t bodyA;
	int32_t bodyB;
	int32_t inUse;
	V3 localAnchorA;
	V3 localAnchorB;
	float length;
	float hertz;
	float dampingRatio;
	V3 localAxisA;
	V3 localAxisB;
	V3 localRefA;
	V3 localRefB;
	int32_t enableLimit;
	float lowerAngle;
	float upperAngle;
	int32_t enableMotor;
	float motorSpeed;
	float maxMotorTorque;
	Q4 relRot0;
	float compliance;
	float lambda;
	float motorLambda;
	uint32_t generation;
};

struct BodySoA
{
	float4* pos;
	float4* rot;
	float4* vel;
	float4* angVel;
	float4* prevPos;
	float4* prevRot;
	float4* prevVel;
	float4* prevAngVel;
	float4* massInv; // invMass, invInertiaLocal.xyz
	float4* iw0;     // invInertiaWorld columns
	float4* iw1;
	float4* iw2;
	float4* force;
	float4* torque;
	float2* sleep; // sleepTime, smoothedEnergy
	uint8_t* state;
	BodyCold* cold;
	// broadphase sidecars
	float4* fatLo;
	float4* fatHi;
	uint8_t* hasFat;
	uint8_t* moved;
	uint8_t* isActive;
	uint8_t* isStable;
	uint8_t* inStableTier;  // stable at the last stable-tier build
	uint8_t* inStableCells; // binned into stable-tier cells at that build
	uint8_t* bFlags;
	// world of each body when the arena packs several worlds (a batch); null
	// when it holds one world
	uint32_t* world;
	int32_t capacity;
};

M3G_D uint32_t worldOfBody(const BodySoA& B, int i) { return B.world != nullptr ? B.world[i] : 0u; }

struct ContactSoA
{
	int2* bodies;
	int32_t* pointCount;
	uint8_t* flags;
	float4* normal; // xyz + friction
	float2* mat;    // restitution, rollingResistance
	float4* cachePosA;
	float4* cacheRotA;
	float4* cachePosB;
	float4* cacheRotB;
	// points, slot-major [slot * capacity + contact]
	float4* pAnchorA; // localAnchorA.xyz, separation
	float4* pAnchorB; // localAnchorB.xyz, id (bits)
	float4* pFricA;   // frictionAnchorA.xyz, lambdaN
	float4* pFricB;   // frictionAnchorB.xyz, lambdaT
	float4* pSlip;    // slipDir.xyz, separationOffset
	float4* pRA;      // rA.xyz, wN
	float4* pRB;      // rB.xyz
	float4* pJA;      // angJA.xyz
	float4* pJB;      // angJB.xyz
	int32_t capacity;
};

// ---- load / store helpers -------------------------------------------------
M3G_HD V3 ld3(const float4& f) { return v3(f.x, f.y, f.z); }
M3G_HD Q4 ldq(const float4& f) { return q4(f.x, f.y, f.z, f.w); }
M3G_HD float4 st3(V3 v, float w = 0.0f) { return make_float4(v.x, v.y, v.z, w); }
M3G_HD float4 stq(Q4 q) { return make_float4(q.x, q.y, q.z, q.w); }

M3G_D M3 loadIW(const BodySoA& B, int i)
{
	M3 m;
	m.cx = ld3(B.iw0[i]);
	m.cy = ld3(B.iw1[i]);
	m.cz = ld3(B.iw2[i]);
	return m;
}
M3G_D void storeIW(const BodySoA& B, int i, const M3& m)
{
	B.iw0[i] = st3(m.cx);
	B.iw1[i] = st3(m.cy);
	B.iw2[i] = st3(m.cz);
}

M3G_D void loadPoint(const ContactSoA& C, int c, int slot, ManifoldPoint& mp)
{
	size_t k = (size_t)slot * (size_t)C.capacity + (size_t)c;
	float4 a = C.pAnchorA[k], b = C.pAnchorB[k], fa = C.pFricA[k], fb = C.pFricB[k], s = C.pSlip[k];
	mp.localAnchorA = ld3(a);
	mp.separation = a.w;
	mp.localAnchorB = ld3(b);
	mp.id = __float_as_uint(b.w);
	mp.frictionAnchorA = ld3(fa);
	mp.lambdaN = fa.w;
	mp.frictionAnchorB = ld3(fb);
	mp.lambdaT = fb.w;
	mp.slipDir = ld3(s);
	mp.separationOffset = s.w;
}
M3G_D void storePoint(const ContactSoA& C, int c, int slot, const ManifoldPoint& mp)
{
	size_t k = (size_t)slot * (size_t)C.capacity + (size_t)c;
	C.pAnchorA[k] = st3(mp.localAnchorA, mp.separation);
	C.pAnchorB[k] = st3(mp.localAnchorB, __uint_as_float(mp.id));
	C.pFricA[k] = st3(mp.frictionAnchorA, mp.lambdaN);
	C.pFricB[k] = st3(mp.frictionAnchorB, mp.lambdaT);
	C.pSlip[k] = st3(mp.slipDir, mp.separationOffset);
}
M3G_D void loadManifold(const ContactSoA& C, int c, Manifold& m)
{
	m.normal = ld3(C.normal[c]);
	m.pointCount = C.pointCount[c];
	for (int s = 0; s < m.pointCount; ++s)
	{
		loadPoint(C, c, s, m.points[s]);
	}
}
M3G_D void storeManifold(const ContactSoA& C, int c, const Manifold& m)
{
	float fr = C.normal[c].w;
	C.normal[c] = st3(m.normal, fr);
	C.pointCount[c] = m.pointCount;
	for (int s = 0; s < m.pointCount; ++s)
	{
		storePoint(C, c, s, m.points[s]);
	}
}
M3G_D size_t pidx(const ContactSoA& C, int c, int slot) { return (size_t)slot * (size_t)C.capacity + (size_t)c; }

M3G_D Xf bodyXf(const BodySoA& B, int i)
{
	Xf xf;
	xf.p = ld3(B.pos[i]);
	xf.q = ldq(B.rot[i]);
	return xf;
}

// WakeBodyInternal (reference src/world.cpp:121-140): awake, timers reset,
// stable tier dirty when the body was asleep; static bodies never wake.
// stableDirty holds one word per world (one word for a single world).
M3G_D void wakeBody(const BodySoA& B, int i, uint32_t* stableDirty)
{
	if (B.cold[i].type == kStatic)
	{
		return;
	}
	if (!(B.state[i] & kStAwake))
	{
		stableDirty[worldOfBody(B, i)] = 1;
	}
	B.state[i] |= kStAwake;
	B.sleep[i] = make_float2(0.0f, 4.0f * kSleepEnergyThresh);
	B.bFlags[i] |= kBFAwake;
}

} // namespace m3g

// XPBD substep element routines (reference src/xpbd.cpp): body integration
// with the implicit gyroscopic step and exponential-map rotation, contact
// preparation (safety re-collision, tunnelling rescue, frozen Jacobians),
// normal projection (serial form and colour-lane form), stiction friction,
// velocity reconstruction, the velocity pass and the joints.
//
// Each routine is called by exactly one GPU thread for one body, contact or
// joint; the kernels guarantee that no other thread touches the same dynamic
// body meanwhile (islands are disjoint, colours are body-disjoint).  Body
// state is read into registers, updated and written back, which is exactly
// the reference's read-modify-write sequence.
#pragma once

#include "m3d_collide.cuh"

namespace m3g
{

#if defined(__CUDA_ARCH__)
// libm's float sinf/cosf/atan2f are evaluated in double precision and rounded
// once; the reference's glibc results agree except for rare last-ulp cases.
M3G_D float dsinf(float x) { return (float)sin((double)x); }
M3G_D float dcosf(float x) { return (float)cos((double)x); }
M3G_D float datan2f(float y, float x) { return (float)atan2((double)y, (double)x); }
#else
inline float dsinf(float x) { return sinf(x); }
inline float dcosf(float x) { return cosf(x); }
inline float datan2f(float y, float x) { return atan2f(y, x); }
#endif

// Per-body state the solver works on, held in registers.
struct BodyDyn
{
	V3 p;
	Q4 q;
	float invMass;
	M3 iw;
};

M3G_D BodyDyn loadDyn(const BodySoA& B, int i)
{
	BodyDyn b;
	b.p = ld3(B.pos[i]);
	b.q = ldq(B.rot[i]);
	b.invMass = B.massInv[i].x;
	b.iw = loadIW(B, i);
	return b;
}
M3G_D void storePose(const BodySoA& B, int i, const BodyDyn& b)
{
	if (b.invMass == 0.0f)
	{
		return; // static / kinematic bodies are shared read-only
	}
	B.pos[i] = st3(b.p);
	B.rot[i] = stq(b.q);
}

// position correction P applied at arm r (reference src/xpbd.cpp:28-41)
M3G_HD void applyPositionCorrection(BodyDyn& b, V3 p, V3 r)
{
	if (b.invMass == 0.0f)
	{
		return;
	}
	b.p = madd(b.p, b.invMass, p);
	V3 dw = mulv(b.iw, cross(r, p));
	Q4 dq = qmul(q4(dw.x, dw.y, dw.z, 0.0f), b.q);
	b.q = qrenormFast(q4(b.q.x + 0.5f * dq.x, b.q.y + 0.5f * dq.y, b.q.z + 0.5f * dq.z, b.q.w + 0.5f * dq.w));
}

// correction of signed magnitude along n with a frozen angular Jacobian
// (reference src/xpbd.cpp:45-58)
M3G_HD void applyAxisCorrection(BodyDyn& b, float dl, V3 n, V3 angJ)
{
	if (b.invMass == 0.0f)
	{
		return;
	}
	b.p = madd(b.p, dl * b.invMass, n);
	V3 dw = scale(dl, angJ);
	Q4 dq = qmul(q4(dw.x, dw.y, dw.z, 0.0f), b.q);
	b.q = qrenormFast(q4(b.q.x + 0.5f * dq.x, b.q.y + 0.5f * dq.y, b.q.z + 0.5f * dq.z, b.q.w + 0.5f * dq.w));
}

M3G_HD float generalizedInvMass(const BodyDyn& b, V3 r, V3 axis)
{
	V3 rn = cross(r, axis);
	return b.invMass + dot(rn, mulv(b.iw, rn));
}

// geometric contact arm for curved shapes, stored anchor for boxes
// (reference src/xpbd.cpp:100-116)
M3G_HD V3 contactArm(const Shape& s, Q4 rot, V3 localAnchor, V3 n, float sign)
{
	switch (s.type)
	{
		case kSphere:
			return scale(sign * s.radius, n);
		case kCapsule:
		{
			float hh = s.halfHeight;
			float axialY = localAnchor.y < -hh ? -hh : (localAnchor.y > hh ? hh : localAnchor.y);
			V3 axis = rotate(rot, v3(0.0f, 1.0f, 0.0f));
			return add(scale(axialY, axis), scale(sign * s.radius, n));
		}
		default:
			return rotate(rot, localAnchor);
	}
}

// ---- body stages ----------------------------------------------------------

// gravity, user force/torque, damping, implicit gyroscopic Newton step,
// position update and exponential-map rotation (reference src/xpbd.cpp:587-705)
M3G_D void integrateBody(const BodySoA& B, int i, float h, V3 gravity)
{
	const BodyCold& cold = B.cold[i];
	if (cold.type != kDynamic)
	{
		return;
	}
	V3 v = ld3(B.vel[i]);
	V3 w = ld3(B.angVel[i]);
	Q4 q = ldq(B.rot[i]);
	V3 x = ld3(B.pos[i]);
	float4 mi = B.massInv[i];
	B.prevVel[i] = st3(v);
	B.prevAngVel[i] = st3(w);

	v = madd(v, h * cold.gravityScale, gravity);
	V3 f = ld3(B.force[i]);
	if (f.x != 0.0f || f.y != 0.0f || f.z != 0.0f)
	{
		v = madd(v, h * mi.x, f);
	}
	V3 tq = ld3(B.torque[i]);
	if (tq.x != 0.0f || tq.y != 0.0f || tq.z != 0.0f)
	{
		M3 iw = loadIW(B, i);
		w = add(w, scale(h, mulv(iw, tq)));
	}
	v = scale(1.0f / (1.0f + h * cold.linearDamping), v);
	w = scale(1.0f / (1.0f + h * cold.angularDamping), w);

	V3 il = v3(mi.y, mi.z, mi.w);
	bool anisotropic = il.x != il.y || il.y != il.z;
	if (anisotropic && il.x > 0.0f && il.y > 0.0f && il.z > 0.0f && len2(w) > 1.0f)
	{
		V3 w0 = invRotate(q, w);
		V3 wl = w0;
		V3 I = v3(1.0f / il.x, 1.0f / il.y, 1.0f / il.z);
		for (int it = 0; it < 1; ++it)
		{
			V3 Iw = v3(I.x * wl.x, I.y * wl.y, I.z * wl.z);
			V3 fr = add(v3(I.x * (wl.x - w0.x), I.y * (wl.y - w0.y), I.z * (wl.z - w0.z)), scale(h, cross(wl, Iw)));
			V3 ex = v3(1.0f, 0.0f, 0.0f), ey = v3(0.0f, 1.0f, 0.0f), ez = v3(0.0f, 0.0f, 1.0f);
			V3 c0 = add(v3(I.x, 0.0f, 0.0f), scale(h, sub(scale(I.x, cross(wl, ex)), cross(Iw, ex))));
			V3 c1 = add(v3(0.0f, I.y, 0.0f), scale(h, sub(scale(I.y, cross(wl, ey)), cross(Iw, ey))));
			V3 c2 = add(v3(0.0f, 0.0f, I.z), scale(h, sub(scale(I.z, cross(wl, ez)), cross(Iw, ez))));
			float det = dot(c0, cross(c1, c2));
			if (fabsf(det) <= 1e-12f)
			{
				break;
			}
			V3 rhs = neg(fr);
			float invDet = 1.0f / det;
			V3 dw = v3(dot(rhs, cross(c1, c2)) * invDet, dot(c0, cross(rhs, c2)) * invDet, dot(c0, cross(c1, rhs)) * invDet);
			wl = add(wl, dw);
		}
		w = rotate(q, wl);
	}

	B.prevPos[i] = st3(x);
	B.prevRot[i] = stq(q);
	x = madd(x, h, v);
	float wlen = len(w);
	if (wlen > 1e-9f)
	{
		float half = 0.5f * h * wlen;
		float sinHalf, cosHalf;
		if (half < 0.02f)
		{
			float h2 = half * half;
			sinHalf = half * (1.0f - h2 * (1.0f / 6.0f));
			cosHalf = 1.0f - h2 * 0.5f;
		}
		else
		{
			sinHalf = dsinf(half);
			cosHalf = dcosf(half);
		}
		float s = sinHalf / wlen;
		Q4 dq = q4(w.x * s, w.y * s, w.z * s, cosHalf);
		q = qrenormFast(qmul(dq, q));
	}
	B.pos[i] = st3(x);
	B.rot[i] = stq(q);
	B.vel[i] = st3(v);
	B.angVel[i] = st3(w);
	storeIW(B, i, invInertiaWorld(q, il));
}

// v from the position delta, w from the exact log map of the rotation delta
// (reference src/xpbd.cpp:865-892)
M3G_D void reconstructBody(const BodySoA& B, int i, float invH)
{
	if (B.cold[i].type != kDynamic)
	{
		return;
	}
	V3 x = ld3(B.pos[i]), x0 = ld3(B.prevPos[i]);
	Q4 q = ldq(B.rot[i]), q0 = ldq(B.prevRot[i]);
	B.vel[i] = st3(scale(invH, sub(x, x0)));
	Q4 dq = qmul(q, qconj(q0));
	float sign = dq.w >= 0.0f ? 1.0f : -1.0f;
	float v2 = dq.x * dq.x + dq.y * dq.y + dq.z * dq.z;
	V3 w;
	if (v2 > 4e-4f)
	{
		float vl = sqrtf(v2);
		float angle = 2.0f * datan2f(vl, fabsf(dq.w));
		w = scale(sign * invH * angle / vl, v3(dq.x, dq.y, dq.z));
	}
	else
	{
		float corr = 1.0f + v2 * (1.0f / 6.0f);
		w = scale(2.0f * invH * sign * corr, v3(dq.x, dq.y, dq.z));
	}
	B.angVel[i] = st3(w);
}

M3G_D void refreshInvInertia(const BodySoA& B, int i)
{
	float4 mi = B.massInv[i];
	storeIW(B, i, invInertiaWorld(ldq(B.rot[i]), v3(mi.y, mi.z, mi.w)));
}

// ---- contacts ---------------------------------------------------------------

// smallest anchor-tracked separation at the current poses
// (reference src/m3d_internal.h:251-268)
M3G_HD float trackedMinSep(Xf xa, Xf xb, const Manifold& m)
{
	if (m.pointCount == 0)
	{
		return 1e30f;
	}
	float mn = 1e30f;
	for (int i = 0; i < m.pointCount; ++i)
	{
		const ManifoldPoint& mp = m.points[i];
		V3 rA = rotate(xa.q, mp.localAnchorA);
		V3 rB = rotate(xb.q, mp.localAnchorB);
		float s = mp.separationOffset + dot(sub(add(xb.p, rB), add(xa.p, rA)), m.normal);
		mn = s < mn ? s : mn;
	}
	return mn;
}

// pose moved beyond 1 mm / ~1 mrad since the cached manifold
// (reference src/m3d_internal.h:231-241)
M3G_HD bool poseChanged(Xf xf, V3 cachePos, Q4 cacheRot)
{
	const float kTolPosSq = 1e-3f * 1e-3f;
	const float kTolHalfAngleSq = 0.25f * 1e-6f;
	if (len2(sub(xf.p, cachePos)) > kTolPosSq)
	{
		return true;
	}
	Q4 d = qmul(xf.q, qconj(cacheRot));
	return d.x * d.x + d.y * d.y + d.z * d.z > kTolHalfAngleSq;
}

// separationOffset = separation - n.(pB + rB - pA - rA) at the generation pose
M3G_HD void setSeparationOffsets(Manifold& m, Xf xa, Xf xb)
{
	for (int p = 0; p < m.pointCount; ++p)
	{
		ManifoldPoint& mp = m.points[p];
		V3 rA = rotate(xa.q, mp.localAnchorA);
		V3 rB = rotate(xb.q, mp.localAnchorB);
		float ref = dot(sub(add(xb.p, rB), add(xa.p, rA)), m.normal);
		mp.separationOffset = mp.separation - ref;
	}
}

// Per-substep preparation of one contact: safety re-collision when a body
// moved > 3 cm or ~5.7 deg since generation, the thin-feature tunnelling
// rescue, then the freeze of arms, Jacobians and normal mass
// (reference src/xpbd.cpp:718-863)
// what prepareContact did to the manifold (differentiation tape)
constexpr int kPrepRegenerated = 2; // regenerated at the current poses
constexpr int kPrepHeld = 4;        // stale, but held by the tunnelling guard

// The stale-manifold half of prepareContact: safety re-collision, tunnelling
// rescue and anchor inheritance (reference src/xpbd.cpp:740-800).  Kept out
// of line: it runs only for contacts whose bodies moved or turned past the
// re-collision thresholds since the manifold was made, and inlining its
// collision code into every solve kernel bloats their hot loops (the serial
// and tiny-island kernels stall on instruction fetch).  Writes the new
// manifold and flags; returns kPrepRegenerated or kPrepHeld.
static __device__ __noinline__ int prepareStaleContact(const BodySoA& B, const ContactSoA& C, int c, float h, Xf xa, Xf xb,
												uint8_t flags, bool hasCache)
{
	int what = 0;
	int2 ab = C.bodies[c];
	const BodyCold& ca = B.cold[ab.x];
	const BodyCold& cb = B.cold[ab.y];
	Manifold oldM, m;
	loadManifold(C, c, oldM);
	m = oldM; // regeneration writes into the existing storage
	V3 va = ld3(B.vel[ab.x]), vb = ld3(B.vel[ab.y]);
	float relSpeed = len(sub(va, vb));
	collideShapes(ca.shape, xa, cb.shape, xb, kSpeculativeBase + h * relSpeed, &m);

	bool keepOld = false;
	bool guard = (flags & kCFTunnelGuard) != 0;
	if (hasCache && oldM.pointCount > 0)
	{
		if (guard)
		{
			keepOld = trackedMinSep(xa, xb, oldM) < -kLinearSlop;
		}
		else
		{
			bool flipOrGone = m.pointCount == 0 || dot(m.normal, oldM.normal) < -0.5f;
			if (flipOrGone)
			{
				V3 dB = cb.type == kDynamic ? sub(xb.p, ld3(B.prevPos[ab.y])) : vzero();
				V3 dA = ca.type == kDynamic ? sub(xa.p, ld3(B.prevPos[ab.x])) : vzero();
				V3 travel = sub(dB, dA);
				float travelLen = len(travel);
				float coreB = cb.shape.type == kBox ? fminf(cb.shape.he.x, fminf(cb.shape.he.y, cb.shape.he.z))
													: cb.shape.radius;
				float minHalfA = ca.shape.type == kBox ? fminf(ca.shape.he.x, fminf(ca.shape.he.y, ca.shape.he.z))
													   : ca.shape.radius;
				float crossSpan = 2.0f * (minHalfA + coreB);
				if (travelLen > 0.04f && travelLen > 0.8f * crossSpan)
				{
					Shape infl = ca.shape;
					if (infl.type == kBox)
					{
						infl.he = add(infl.he, v3(coreB, coreB, coreB));
					}
					else
					{
						infl.radius += coreB;
					}
					float backup = 2.0f * coreB + 0.02f;
					V3 dir = scale(1.0f / travelLen, travel);
					V3 origin = sub(sub(xb.p, dB), scale(backup, dir));
					V3 seg = add(travel, scale(backup, dir));
					float fhit;
					V3 nhit;
					keepOld = rayCastShape(infl, xa, origin, seg, &fhit, &nhit);
				}
			}
		}
		guard = keepOld;
	}
	if (keepOld)
	{
		m = oldM; // cache pose intentionally not refreshed
		what = kPrepHeld;
	}
	else
	{
		what = kPrepRegenerated;
		inheritAnchors(oldM, m, ca.shape.type == kBox && cb.shape.type == kBox, xa, xb);
		hasCache = true;
		C.cachePosA[c] = st3(xa.p);
		C.cacheRotA[c] = stq(xa.q);
		C.cachePosB[c] = st3(xb.p);
		C.cacheRotB[c] = stq(xb.q);
		setSeparationOffsets(m, xa, xb);
	}
	storeManifold(C, c, m);
	uint8_t nf = flags;
	nf = guard ? (uint8_t)(nf | kCFTunnelGuard) : (uint8_t)(nf & ~kCFTunnelGuard);
	nf = hasCache ? (uint8_t)(nf | kCFHasCache) : nf;
	C.flags[c] = nf;
	return what;
}

M3G_D int prepareContact(const BodySoA& B, const ContactSoA& C, int c, float h)
{
	int what = 0;
	int2 ab = C.bodies[c];
	const BodyCold& ca = B.cold[ab.x];
	const BodyCold& cb = B.cold[ab.y];
	Xf xa = bodyXf(B, ab.x), xb = bodyXf(B, ab.y);
	uint8_t flags = C.flags[c];
	bool hasCache = (flags & kCFHasCache) != 0;

	bool stale = !hasCache;
	if (!stale)
	{
		const float kReCollidePosSq = 0.03f * 0.03f;
		const float kReCollideHalfAngSq = 0.05f * 0.05f;
		V3 cpa = ld3(C.cachePosA[c]), cpb = ld3(C.cachePosB[c]);
		if (len2(sub(xa.p, cpa)) > kReCollidePosSq || len2(sub(xb.p, cpb)) > kReCollidePosSq)
		{
			stale = true;
		}
		else
		{
			Q4 da = qmul(xa.q, qconj(ldq(C.cacheRotA[c])));
			Q4 db = qmul(xb.q, qconj(ldq(C.cacheRotB[c])));
			stale = da.x * da.x + da.y * da.y + da.z * da.z > kReCollideHalfAngSq ||
					db.x * db.x + db.y * db.y + db.z * db.z > kReCollideHalfAngSq;
		}
	}

	if (stale)
	{
		what = prepareStaleContact(B, C, c, h, xa, xb, flags, hasCache);
	}
	int pointCount = C.pointCount[c];
	V3 n = ld3(C.normal[c]);
	float invMassA = B.massInv[ab.x].x, invMassB = B.massInv[ab.y].x;
	M3 iwA = loadIW(B, ab.x), iwB = loadIW(B, ab.y);
	for (int s = 0; s < pointCount; ++s)
	{
		size_t k = pidx(C, c, s);
		V3 la = ld3(C.pAnchorA[k]);
		V3 lb = ld3(C.pAnchorB[k]);
		V3 rA = contactArm(ca.shape, xa.q, la, n, 1.0f);
		V3 rB = contactArm(cb.shape, xb.q, lb, n, -1.0f);
		V3 crossA = cross(rA, n);
		V3 crossB = cross(rB, n);
		V3 jA = mulv(iwA, crossA);
		V3 jB = mulv(iwB, crossB);
		float wN = invMassA + invMassB + dot(crossA, jA) + dot(crossB, jB);
		float4 fa = C.pFricA[k];
		fa.w = 0.0f; // lambdaN
		C.pFricA[k] = fa;
		float4 fb = C.pFricB[k];
		fb.w = 0.0f; // lambdaT
		C.pFricB[k] = fb;
		C.pRA[k] = st3(rA, wN);
		C.pRB[k] = st3(rB);
		C.pJA[k] = st3(jA);
		C.pJB[k] = st3(jB);
	}
	return what;
}

// Gauss-Seidel normal projection of one contact, serial-island form
// (reference src/xpbd.cpp:122-163)
M3G_D void solveContactNormals(const BodySoA& B, const ContactSoA& C, int c, float maxCorrection)
{
	int2 ab = C.bodies[c];
	int pc = C.pointCount[c];
	if (pc == 0)
	{
		return;
	}
	BodyDyn a = loadDyn(B, ab.x), b = loadDyn(B, ab.y);
	V3 n = ld3(C.normal[c]);
	for (int s = 0; s < pc; ++s)
	{
		size_t k = pidx(C, c, s);
		float wN = C.pRA[k].w;
		if (wN <= 0.0f)
		{
			continue;
		}
		V3 rA = rotate(a.q, ld3(C.pAnchorA[k]));
		V3 rB = rotate(b.q, ld3(C.pAnchorB[k]));
		float sep = C.pSlip[k].w + dot(sub(add(b.p, rB), add(a.p, rA)), n);
		if (sep >= 0.0f)
		{
			continue;
		}
		if (sep < -maxCorrection)
		{
			sep = -maxCorrection;
		}
		float dl = -sep / wN;
		float4 fa = C.pFricA[k];
		fa.w += dl;
		C.pFricA[k] = fa;
		applyAxisCorrection(b, dl, n, ld3(C.pJB[k]));
		applyAxisCorrection(a, -dl, n, ld3(C.pJA[k]));
	}
	storePose(B, ab.x, a);
	storePose(B, ab.y, b);
}

// solveContactNormals with the data of every point loaded before the first
// correction: none of it depends on the corrections, and issuing the loads
// together costs the contact a few memory round trips instead of two per
// point.  Same arithmetic, point by point.  It needs ~100 more registers, so
// only the kernel whose sweeps are one level of contacts at a time on one CTA
// (the overflow bucket of giant islands) uses it.
M3G_D void solveContactNormalsPrefetched(const BodySoA& B, const ContactSoA& C, int c, float maxCorrection)
{
	int2 ab = C.bodies[c];
	int pc = C.pointCount[c];
	if (pc == 0)
	{
		return;
	}
	float wN[4], sepOff[4], lamN[4];
	V3 anA[4], anB[4], jA[4], jB[4];
#pragma unroll
	for (int s = 0; s < 4; ++s)
	{
		if (s < pc)
		{
			size_t k = pidx(C, c, s);
			wN[s] = C.pRA[k].w;
			anA[s] = ld3(C.pAnchorA[k]);
			anB[s] = ld3(C.pAnchorB[k]);
			sepOff[s] = C.pSlip[k].w;
			lamN[s] = C.pFricA[k].w;
			jA[s] = ld3(C.pJA[k]);
			jB[s] = ld3(C.pJB[k]);
		}
	}
	BodyDyn a = loadDyn(B, ab.x), b = loadDyn(B, ab.y);
	V3 n = ld3(C.normal[c]);
#pragma unroll
	for (int s = 0; s < 4; ++s)
	{
		if (s >= pc)
		{
			break;
		}
		if (wN[s] <= 0.0f)
		{
			continue;
		}
		V3 rA = rotate(a.q, anA[s]);
		V3 rB = rotate(b.q, anB[s]);
		float sep = sepOff[s] + dot(sub(add(b.p, rB), add(a.p, rA)), n);
		if (sep >= 0.0f)
		{
			continue;
		}
		if (sep < -maxCorrection)
		{
			sep = -maxCorrection;
		}
		float dl = -sep / wN[s];
		C.pFricA[pidx(C, c, s)].w = lamN[s] + dl;
		applyAxisCorrection(b, dl, n, jB[s]);
		applyAxisCorrection(a, -dl, n, jA[s]);
	}
	storePose(B, ab.x, a);
	storePose(B, ab.y, b);
}

// Normal projection of one contact as one lane of a colour packet
// (reference src/xpbd.cpp:1047-1141).  The lane sweeps `maxPoints` slots -
// the largest point count among the 8 contacts of its packet - and slots past
// its own point count still run with a zero gate: the fast quaternion
// renormalisation of both lane bodies happens on every slot, as in the
// reference's branchless 8-wide loop.  Lambdas accumulate straight into the
// manifold points (the reference's packet copy is flushed there unchanged).
M3G_D void solvePacketLane(const BodySoA& B, const ContactSoA& C, int c, int maxPoints, float maxCorrection)
{
	int2 ab = C.bodies[c];
	int pc = C.pointCount[c];
	float imA = B.massInv[ab.x].x, imB = B.massInv[ab.y].x;
	V3 pa = ld3(B.pos[ab.x]), pb = ld3(B.pos[ab.y]);
	Q4 qa = ldq(B.rot[ab.x]), qb = ldq(B.rot[ab.y]);
	V3 n = ld3(C.normal[c]);
	for (int s = 0; s < maxPoints; ++s)
	{
		bool on = s < pc;
		V3 la = vzero(), lb = vzero(), jA = vzero(), jB = vzero();
		float sepOff = 0.0f, invW = 1.0f, active = 0.0f;
		size_t k = pidx(C, c, s);
		if (on)
		{
			la = ld3(C.pAnchorA[k]);
			lb = ld3(C.pAnchorB[k]);
			sepOff = C.pSlip[k].w;
			float wN = C.pRA[k].w;
			invW = wN > 0.0f ? 1.0f / wN : 1.0f;
			jA = ld3(C.pJA[k]);
			jB = ld3(C.pJB[k]);
			active = 1.0f;
		}
		// anchors rotated by the current lane rotations
		float tx = 2.0f * (qa.y * la.z - qa.z * la.y);
		float ty = 2.0f * (qa.z * la.x - qa.x * la.z);
		float tz = 2.0f * (qa.x * la.y - qa.y * la.x);
		float rax = la.x + qa.w * tx + (qa.y * tz - qa.z * ty);
		float ray = la.y + qa.w * ty + (qa.z * tx - qa.x * tz);
		float raz = la.z + qa.w * tz + (qa.x * ty - qa.y * tx);
		tx = 2.0f * (qb.y * lb.z - qb.z * lb.y);
		ty = 2.0f * (qb.z * lb.x - qb.x * lb.z);
		tz = 2.0f * (qb.x * lb.y - qb.y * lb.x);
		float rbx = lb.x + qb.w * tx + (qb.y * tz - qb.z * ty);
		float rby = lb.y + qb.w * ty + (qb.z * tx - qb.x * tz);
		float rbz = lb.z + qb.w * tz + (qb.x * ty - qb.y * tx);

		float sep = sepOff + (pb.x + rbx - pa.x - rax) * n.x + (pb.y + rby - pa.y - ray) * n.y +
					(pb.z + rbz - pa.z - raz) * n.z;
		float gate = sep < 0.0f ? active : 0.0f;
		float capped = sep < -maxCorrection ? -maxCorrection : sep;
		float dL = -capped * invW * gate;
		if (on)
		{
			float4 fa = C.pFricA[k];
			fa.w += dL;
			C.pFricA[k] = fa;
		}

		pb.x += dL * imB * n.x;
		pb.y += dL * imB * n.y;
		pb.z += dL * imB * n.z;
		pa.x -= dL * imA * n.x;
		pa.y -= dL * imA * n.y;
		pa.z -= dL * imA * n.z;

		float dwx = dL * jB.x, dwy = dL * jB.y, dwz = dL * jB.z;
		float dqx = dwx * qb.w + dwy * qb.z - dwz * qb.y;
		float dqy = -dwx * qb.z + dwy * qb.w + dwz * qb.x;
		float dqz = dwx * qb.y - dwy * qb.x + dwz * qb.w;
		float dqw = -(dwx * qb.x + dwy * qb.y + dwz * qb.z);
		float x = qb.x + 0.5f * dqx, y = qb.y + 0.5f * dqy, z = qb.z + 0.5f * dqz, w = qb.w + 0.5f * dqw;
		float sc = 1.5f - 0.5f * (x * x + y * y + z * z + w * w);
		qb = q4(x * sc, y * sc, z * sc, w * sc);

		dwx = -dL * jA.x;
		dwy = -dL * jA.y;
		dwz = -dL * jA.z;
		dqx = dwx * qa.w + dwy * qa.z - dwz * qa.y;
		dqy = -dwx * qa.z + dwy * qa.w + dwz * qa.x;
		dqz = dwx * qa.y - dwy * qa.x + dwz * qa.w;
		dqw = -(dwx * qa.x + dwy * qa.y + dwz * qa.z);
		x = qa.x + 0.5f * dqx;
		y = qa.y + 0.5f * dqy;
		z = qa.z + 0.5f * dqz;
		w = qa.w + 0.5f * dqw;
		sc = 1.5f - 0.5f * (x * x + y * y + z * z + w * w);
		qa = q4(x * sc, y * sc, z * sc, w * sc);
	}
	if (imA > 0.0f)
	{
		B.pos[ab.x] = st3(pa);
		B.rot[ab.x] = stq(qa);
	}
	if (imB > 0.0f)
	{
		B.pos[ab.y] = st3(pb);
		B.rot[ab.y] = stq(qb);
	}
}

// Positional stiction toward persistent anchors, box-box only, once per
// substep (reference src/xpbd.cpp:172-269)
M3G_D void applyContactFriction(const BodySoA& B, const ContactSoA& C, int c)
{
	int2 ab = C.bodies[c];
	const BodyCold& ca = B.cold[ab.x];
	const BodyCold& cb = B.cold[ab.y];
	if (ca.shape.type != kBox || cb.shape.type != kBox)
	{
		return;
	}
	int pc = C.pointCount[c];
	if (pc == 0)
	{
		return;
	}
	float4 nf = C.normal[c];
	V3 n = ld3(nf);
	float friction = nf.w;
	{
		const float kStictionMaxSpeedSq = 0.1f * 0.1f;
		size_t k0 = pidx(C, c, 0);
		V3 rA0 = ld3(C.pRA[k0]), rB0 = ld3(C.pRB[k0]);
		V3 va = ld3(B.vel[ab.x]), wa = ld3(B.angVel[ab.x]);
		V3 vb = ld3(B.vel[ab.y]), wb = ld3(B.angVel[ab.y]);
		V3 vrel = sub(add(vb, cross(wb, rB0)), add(va, cross(wa, rA0)));
		V3 vt = sub(vrel, scale(dot(vrel, n), n));
		if (len2(vt) > kStictionMaxSpeedSq)
		{
			for (int s = 0; s < pc; ++s)
			{
				size_t k = pidx(C, c, s);
				float4 fa = C.pFricA[k], fb = C.pFricB[k];
				float4 la = C.pAnchorA[k], lb = C.pAnchorB[k];
				C.pFricA[k] = make_float4(la.x, la.y, la.z, fa.w);
				C.pFricB[k] = make_float4(lb.x, lb.y, lb.z, fb.w);
			}
			return;
		}
	}
	BodyDyn a = loadDyn(B, ab.x), b = loadDyn(B, ab.y);
	for (int s = 0; s < pc; ++s)
	{
		size_t k = pidx(C, c, s);
		float4 fa = C.pFricA[k], fb = C.pFricB[k];
		float lambdaN = fa.w;
		if (lambdaN <= 0.0f)
		{
			continue;
		}
		V3 rA = rotate(a.q, ld3(fa));
		V3 rB = rotate(b.q, ld3(fb));
		V3 gap = sub(add(b.p, rB), add(a.p, rA));
		V3 dpt = sub(gap, scale(dot(gap, n), n));
		float lt = len(dpt);
		if (lt <= 1e-9f)
		{
			continue;
		}
		V3 t = scale(1.0f / lt, dpt);
		float wt = generalizedInvMass(a, rA, t) + generalizedInvMass(b, rB, t);
		if (wt <= 0.0f)
		{
			continue;
		}
		float needed = kFrictionRelaxation * (lt / wt);
		float allowed = friction * lambdaN - fb.w;
		if (allowed <= 0.0f)
		{
			continue;
		}
		float dL = needed < allowed ? needed : allowed;
		fb.w += dL;
		V3 pt = scale(dL, t);
		applyPositionCorrection(b, neg(pt), rB);
		applyPositionCorrection(a, pt, rA);
		if (needed > 2.0f * allowed)
		{
			float4 la = C.pAnchorA[k], lb = C.pAnchorB[k];
			fa = make_float4(la.x, la.y, la.z, fa.w);
			fb = make_float4(lb.x, lb.y, lb.z, fb.w);
			C.pFricA[k] = fa;
		}
		C.pFricB[k] = fb;
	}
	storePose(B, ab.x, a);
	storePose(B, ab.y, b);
}

// applyContactFriction with every point's records loaded up front (see
// solveContactVelocityPrefetched): same arithmetic, for the overflow levels of
// giant islands.
M3G_D void applyContactFrictionPrefetched(const BodySoA& B, const ContactSoA& C, int c)
{
	int2 ab = C.bodies[c];
	const BodyCold& ca = B.cold[ab.x];
	const BodyCold& cb = B.cold[ab.y];
	if (ca.shape.type != kBox || cb.shape.type != kBox)
	{
		return;
	}
	int pc = C.pointCount[c];
	if (pc == 0)
	{
		return;
	}
	float4 nf = C.normal[c];
	V3 n = ld3(nf);
	float friction = nf.w;
	// every point's friction and local anchors, loaded before the first
	// update (each point writes only its own records)
	float4 faP[4], fbP[4], laP[4], lbP[4];
#pragma unroll
	for (int s = 0; s < 4; ++s)
	{
		if (s < pc)
		{
			size_t k = pidx(C, c, s);
			faP[s] = C.pFricA[k];
			fbP[s] = C.pFricB[k];
			laP[s] = C.pAnchorA[k];
			lbP[s] = C.pAnchorB[k];
		}
	}
	{
		const float kStictionMaxSpeedSq = 0.1f * 0.1f;
		size_t k0 = pidx(C, c, 0);
		V3 rA0 = ld3(C.pRA[k0]), rB0 = ld3(C.pRB[k0]);
		V3 va = ld3(B.vel[ab.x]), wa = ld3(B.angVel[ab.x]);
		V3 vb = ld3(B.vel[ab.y]), wb = ld3(B.angVel[ab.y]);
		V3 vrel = sub(add(vb, cross(wb, rB0)), add(va, cross(wa, rA0)));
		V3 vt = sub(vrel, scale(dot(vrel, n), n));
		if (len2(vt) > kStictionMaxSpeedSq)
		{
#pragma unroll
			for (int s = 0; s < 4; ++s)
			{
				if (s >= pc)
				{
					break;
				}
				size_t k = pidx(C, c, s);
				float4 fa = faP[s], fb = fbP[s];
				float4 la = laP[s], lb = lbP[s];
				C.pFricA[k] = make_float4(la.x, la.y, la.z, fa.w);
				C.pFricB[k] = make_float4(lb.x, lb.y, lb.z, fb.w);
			}
			return;
		}
	}
	BodyDyn a = loadDyn(B, ab.x), b = loadDyn(B, ab.y);
#pragma unroll
	for (int s = 0; s < 4; ++s)
	{
		if (s >= pc)
		{
			break;
		}
		size_t k = pidx(C, c, s);
		float4 fa = faP[s], fb = fbP[s];
		float lambdaN = fa.w;
		if (lambdaN <= 0.0f)
		{
			continue;
		}
		V3 rA = rotate(a.q, ld3(fa));
		V3 rB = rotate(b.q, ld3(fb));
		V3 gap = sub(add(b.p, rB), add(a.p, rA));
		V3 dpt = sub(gap, scale(dot(gap, n), n));
		float lt = len(dpt);
		if (lt <= 1e-9f)
		{
			continue;
		}
		V3 t = scale(1.0f / lt, dpt);
		float wt = generalizedInvMass(a, rA, t) + generalizedInvMass(b, rB, t);
		if (wt <= 0.0f)
		{
			continue;
		}
		float needed = kFrictionRelaxation * (lt / wt);
		float allowed = friction * lambdaN - fb.w;
		if (allowed <= 0.0f)
		{
			continue;
		}
		float dL = needed < allowed ? needed : allowed;
		fb.w += dL;
		V3 pt = scale(dL, t);
		applyPositionCorrection(b, neg(pt), rB);
		applyPositionCorrection(a, pt, rA);
		if (needed > 2.0f * allowed)
		{
			float4 la = laP[s], lb = lbP[s];
			fa = make_float4(la.x, la.y, la.z, fa.w);
			fb = make_float4(lb.x, lb.y, lb.z, fb.w);
			C.pFricA[k] = fa;
		}
		C.pFricB[k] = fb;
	}
	storePose(B, ab.x, a);
	storePose(B, ab.y, b);
}

// Velocity pass: Coulomb-capped dynamic friction with the coherence test,
// restitution against the pre-substep normal velocity, the unconditional
// normal-velocity fix and rolling resistance (reference src/xpbd.cpp:275-407)
M3G_D void solveContactVelocity(const BodySoA& B, const ContactSoA& C, int c, float h, float gravityLen)
{
	int2 ab = C.bodies[c];
	int pc = C.pointCount[c];
	const BodyCold& ca = B.cold[ab.x];
	const BodyCold& cb = B.cold[ab.y];
	float4 nf = C.normal[c];
	V3 n = ld3(nf);
	float friction = nf.w;
	float2 mat = C.mat[c];
	bool curved = (C.flags[c] & kCFCurved) != 0;
	float invH = h > 0.0f ? 1.0f / h : 0.0f;
	float lambdaNTotal = 0.0f;

	float imA = B.massInv[ab.x].x, imB = B.massInv[ab.y].x;
	M3 iwA = loadIW(B, ab.x), iwB = loadIW(B, ab.y);
	Q4 qa = ldq(B.rot[ab.x]), qb = ldq(B.rot[ab.y]);
	V3 va = ld3(B.vel[ab.x]), wa = ld3(B.angVel[ab.x]);
	V3 vb = ld3(B.vel[ab.y]), wb = ld3(B.angVel[ab.y]);
	V3 pva = ld3(B.prevVel[ab.x]), pwa = ld3(B.prevAngVel[ab.x]);
	V3 pvb = ld3(B.prevVel[ab.y]), pwb = ld3(B.prevAngVel[ab.y]);
	BodyDyn ga, gb; // for generalised masses
	ga.invMass = imA;
	ga.iw = iwA;
	gb.invMass = imB;
	gb.iw = iwB;

	for (int s = 0; s < pc; ++s)
	{
		size_t k = pidx(C, c, s);
		float lambdaN = C.pFricA[k].w;
		if (lambdaN <= 0.0f)
		{
			continue;
		}
		float4 ra4 = C.pRA[k];
		V3 rAf, rBf;
		if (curved)
		{
			rAf = contactArm(ca.shape, qa, ld3(C.pAnchorA[k]), n, 1.0f);
			rBf = contactArm(cb.shape, qb, ld3(C.pAnchorB[k]), n, -1.0f);
		}
		else
		{
			rAf = ld3(ra4);
			rBf = ld3(C.pRB[k]);
		}
		V3 vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		float vn = dot(vrel, n);
		V3 vt = sub(vrel, scale(vn, n));
		float vtLen = len(vt);
		if (vtLen > 1e-9f)
		{
			V3 t = scale(1.0f / vtLen, vt);
			float wt = generalizedInvMass(ga, rAf, t) + generalizedInvMass(gb, rBf, t);
			if (wt > 0.0f)
			{
				const float kStaticSlipSpeed = 0.08f;
				float4 sl = C.pSlip[k];
				bool coherent = dot(t, ld3(sl)) > 0.7f;
				float pStop = vtLen / wt;
				float pMax = friction * lambdaN * invH;
				float P = !coherent && vtLen < kStaticSlipSpeed ? pStop : (pStop < pMax ? pStop : pMax);
				C.pSlip[k] = st3(t, sl.w);
				V3 p = scale(-P, t);
				if (imB != 0.0f)
				{
					vb = madd(vb, imB, p);
					wb = add(wb, mulv(iwB, cross(rBf, p)));
				}
				if (imA != 0.0f)
				{
					V3 pn = neg(p);
					va = madd(va, imA, pn);
					wa = add(wa, mulv(iwA, cross(rAf, pn)));
				}
			}
		}
		V3 vrelPrev = sub(add(pvb, cross(pwb, rBf)), add(pva, cross(pwa, rAf)));
		float vnPrev = dot(vrelPrev, n);
		float e = fabsf(vnPrev) > 2.0f * gravityLen * h ? mat.x : 0.0f;
		vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		vn = dot(vrel, n);
		float target = -e * vnPrev;
		target = target > 0.0f ? target : 0.0f;
		float wN = ra4.w;
		if (wN > 0.0f)
		{
			float j = (target - vn) / wN;
			if (imB != 0.0f)
			{
				vb = madd(vb, j * imB, n);
				wb = madd(wb, j, ld3(C.pJB[k]));
			}
			if (imA != 0.0f)
			{
				float mj = -j;
				va = madd(va, mj * imA, n);
				wa = madd(wa, mj, ld3(C.pJA[k]));
			}
		}
		lambdaNTotal += lambdaN > 0.0f ? lambdaN : 0.0f;
	}

	float rolling = mat.y;
	if (rolling > 0.0f && lambdaNTotal > 0.0f)
	{
		V3 wrel = sub(wb, wa);
		V3 wroll = sub(wrel, scale(dot(wrel, n), n));
		float wl = len(wroll);
		if (wl > 1e-6f)
		{
			V3 axis = scale(1.0f / wl, wroll);
			float kk = dot(axis, mulv(iwA, axis)) + dot(axis, mulv(iwB, axis));
			if (kk > 1e-12f)
			{
				float maxDw = rolling * lambdaNTotal * invH * kk;
				float dw = maxDw < wl ? maxDw : wl;
				V3 angImp = scale(dw / kk, axis);
				wb = sub(wb, mulv(iwB, angImp));
				wa = add(wa, mulv(iwA, angImp));
			}
		}
	}
	// the reference writes rolling resistance into static bodies too, but their
	// inverse inertia is zero, so the write is a no-op; skip it
	if (imA != 0.0f || ca.type == kDynamic)
	{
		B.vel[ab.x] = st3(va);
		B.angVel[ab.x] = st3(wa);
	}
	if (imB != 0.0f || cb.type == kDynamic)
	{
		B.vel[ab.y] = st3(vb);
		B.angVel[ab.y] = st3(wb);
	}
}

// solveContactVelocity with the data of every point loaded before the first
// update: a contact costs a few memory round trips instead of two per point.
// Same arithmetic, point by point; ~90 more registers, so only the overflow
// levels of giant islands (one level of contacts at a time on one CTA) use it.
M3G_D void solveContactVelocityPrefetched(const BodySoA& B, const ContactSoA& C, int c, float h, float gravityLen)
{
	int2 ab = C.bodies[c];
	int pc = C.pointCount[c];
	const BodyCold& ca = B.cold[ab.x];
	const BodyCold& cb = B.cold[ab.y];
	float4 nf = C.normal[c];
	V3 n = ld3(nf);
	float friction = nf.w;
	float2 mat = C.mat[c];
	bool curved = (C.flags[c] & kCFCurved) != 0;
	float invH = h > 0.0f ? 1.0f / h : 0.0f;
	float lambdaNTotal = 0.0f;

	float imA = B.massInv[ab.x].x, imB = B.massInv[ab.y].x;
	M3 iwA = loadIW(B, ab.x), iwB = loadIW(B, ab.y);
	Q4 qa = ldq(B.rot[ab.x]), qb = ldq(B.rot[ab.y]);
	V3 va = ld3(B.vel[ab.x]), wa = ld3(B.angVel[ab.x]);
	V3 vb = ld3(B.vel[ab.y]), wb = ld3(B.angVel[ab.y]);
	V3 pva = ld3(B.prevVel[ab.x]), pwa = ld3(B.prevAngVel[ab.x]);
	V3 pvb = ld3(B.prevVel[ab.y]), pwb = ld3(B.prevAngVel[ab.y]);
	BodyDyn ga, gb; // for generalised masses
	ga.invMass = imA;
	ga.iw = iwA;
	gb.invMass = imB;
	gb.iw = iwB;

	// every point's data is loaded before the first update: none of it
	// depends on the updates (each point writes only its own slip direction)
	float lamP[4];
	float4 raP[4], slP[4];
	V3 rbP[4], aaP[4], jaP[4], jbP[4];
#pragma unroll
	for (int s = 0; s < 4; ++s)
	{
		if (s < pc)
		{
			size_t k = pidx(C, c, s);
			lamP[s] = C.pFricA[k].w;
			raP[s] = C.pRA[k];
			rbP[s] = curved ? ld3(C.pAnchorB[k]) : ld3(C.pRB[k]);
			aaP[s] = curved ? ld3(C.pAnchorA[k]) : vzero();
			slP[s] = C.pSlip[k];
			jaP[s] = ld3(C.pJA[k]);
			jbP[s] = ld3(C.pJB[k]);
		}
	}
#pragma unroll
	for (int s = 0; s < 4; ++s)
	{
		if (s >= pc)
		{
			break;
		}
		size_t k = pidx(C, c, s);
		float lambdaN = lamP[s];
		if (lambdaN <= 0.0f)
		{
			continue;
		}
		float4 ra4 = raP[s];
		V3 rAf, rBf;
		if (curved)
		{
			rAf = contactArm(ca.shape, qa, aaP[s], n, 1.0f);
			rBf = contactArm(cb.shape, qb, rbP[s], n, -1.0f);
		}
		else
		{
			rAf = ld3(ra4);
			rBf = rbP[s];
		}
		V3 vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		float vn = dot(vrel, n);
		V3 vt = sub(vrel, scale(vn, n));
		float vtLen = len(vt);
		if (vtLen > 1e-9f)
		{
			V3 t = scale(1.0f / vtLen, vt);
			float wt = generalizedInvMass(ga, rAf, t) + generalizedInvMass(gb, rBf, t);
			if (wt > 0.0f)
			{
				const float kStaticSlipSpeed = 0.08f;
				float4 sl = slP[s];
				bool coherent = dot(t, ld3(sl)) > 0.7f;
				float pStop = vtLen / wt;
				float pMax = friction * lambdaN * invH;
				float P = !coherent && vtLen < kStaticSlipSpeed ? pStop : (pStop < pMax ? pStop : pMax);
				C.pSlip[k] = st3(t, sl.w);
				V3 p = scale(-P, t);
				if (imB != 0.0f)
				{
					vb = madd(vb, imB, p);
					wb = add(wb, mulv(iwB, cross(rBf, p)));
				}
				if (imA != 0.0f)
				{
					V3 pn = neg(p);
					va = madd(va, imA, pn);
					wa = add(wa, mulv(iwA, cross(rAf, pn)));
				}
			}
		}
		V3 vrelPrev = sub(add(pvb, cross(pwb, rBf)), add(pva, cross(pwa, rAf)));
		float vnPrev = dot(vrelPrev, n);
		float e = fabsf(vnPrev) > 2.0f * gravityLen * h ? mat.x : 0.0f;
		vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		vn = dot(vrel, n);
		float target = -e * vnPrev;
		target = target > 0.0f ? target : 0.0f;
		float wN = ra4.w;
		if (wN > 0.0f)
		{
			float j = (target - vn) / wN;
			if (imB != 0.0f)
			{
				vb = madd(vb, j * imB, n);
				wb = madd(wb, j, jbP[s]);
			}
			if (imA != 0.0f)
			{
				float mj = -j;
				va = madd(va, mj * imA, n);
				wa = madd(wa, mj, jaP[s]);
			}
		}
		lambdaNTotal += lambdaN > 0.0f ? lambdaN : 0.0f;
	}

	float rolling = mat.y;
	if (rolling > 0.0f && lambdaNTotal > 0.0f)
	{
		V3 wrel = sub(wb, wa);
		V3 wroll = sub(wrel, scale(dot(wrel, n), n));
		float wl = len(wroll);
		if (wl > 1e-6f)
		{
			V3 axis = scale(1.0f / wl, wroll);
			float kk = dot(axis, mulv(iwA, axis)) + dot(axis, mulv(iwB, axis));
			if (kk > 1e-12f)
			{
				float maxDw = rolling * lambdaNTotal * invH * kk;
				float dw = maxDw < wl ? maxDw : wl;
				V3 angImp = scale(dw / kk, axis);
				wb = sub(wb, mulv(iwB, angImp));
				wa = add(wa, mulv(iwA, angImp));
			}
		}
	}
	// the reference writes rolling resistance into static bodies too, but their
	// inverse inertia is zero, so the write is a no-op; skip it
	if (imA != 0.0f || ca.type == kDynamic)
	{
		B.vel[ab.x] = st3(va);
		B.angVel[ab.x] = st3(wa);
	}
	if (imB != 0.0f || cb.type == kDynamic)
	{
		B.vel[ab.y] = st3(vb);
		B.angVel[ab.y] = st3(wb);
	}
}

// ---- joints (reference src/xpbd.cpp:413-581) ---------------------------------

M3G_HD float hingeAngle(Q4 qa, Q4 qb, const JointRec& j)
{
	V3 axis = rotate(qa, j.localAxisA);
	V3 refA = rotate(qa, j.localRefA);
	V3 refB = rotate(qb, j.localRefB);
	float s = dot(axis, cross(refA, refB));
	float c = dot(refA, refB);
	return datan2f(s, c);
}

M3G_D void prepareJoint(const BodySoA& B, JointRec& j)
{
	j.compliance = 0.0f;
	if (j.type == kJointDistance && j.hertz > 0.0f)
	{
		BodyDyn a = loadDyn(B, j.bodyA), b = loadDyn(B, j.bodyB);
		V3 rA = rotate(a.q, j.localAnchorA);
		V3 rB = rotate(b.q, j.localAnchorB);
		V3 d = sub(add(b.p, rB), add(a.p, rA));
		V3 u = normalize(d);
		float w = generalizedInvMass(a, rA, u) + generalizedInvMass(b, rB, u);
		if (w > 0.0f)
		{
			float meff = 1.0f / w;
			float omega = 2.0f * 3.14159265358979323846f * j.hertz;
			float k = meff * omega * omega;
			j.compliance = k > 0.0f ? 1.0f / k : 0.0f;
		}
	}
}

M3G_HD void applyAngularCorrection(BodyDyn& a, BodyDyn& b, V3 corr)
{
	float theta = len(corr);
	if (theta < 1e-9f)
	{
		return;
	}
	V3 n = scale(1.0f / theta, corr);
	float wA = a.invMass != 0.0f ? dot(n, mulv(a.iw, n)) : 0.0f;
	float wB = b.invMass != 0.0f ? dot(n, mulv(b.iw, n)) : 0.0f;
	float denom = wA + wB;
	if (denom <= 0.0f)
	{
		return;
	}
	float lambda = theta / denom;
	V3 p = scale(lambda, n);
	if (a.invMass != 0.0f)
	{
		V3 dw = mulv(a.iw, p);
		Q4 dq = qmul(q4(dw.x, dw.y, dw.z, 0.0f), a.q);
		a.q = qrenormFast(q4(a.q.x + 0.5f * dq.x, a.q.y + 0.5f * dq.y, a.q.z + 0.5f * dq.z, a.q.w + 0.5f * dq.w));
	}
	if (b.invMass != 0.0f)
	{
		V3 dw = mulv(b.iw, p);
		Q4 dq = qmul(q4(-dw.x, -dw.y, -dw.z, 0.0f), b.q);
		b.q = qrenormFast(q4(b.q.x + 0.5f * dq.x, b.q.y + 0.5f * dq.y, b.q.z + 0.5f * dq.z, b.q.w + 0.5f * dq.w));
	}
}

M3G_D void solveJointPosition(const BodySoA& B, JointRec& j, float h)
{
	BodyDyn a = loadDyn(B, j.bodyA), b = loadDyn(B, j.bodyB);
	if (j.type == kJointHinge)
	{
		V3 axisA = rotate(a.q, j.localAxisA);
		V3 axisB = rotate(b.q, j.localAxisB);
		applyAngularCorrection(a, b, cross(axisA, axisB));
		if (j.enableLimit)
		{
			float phi = hingeAngle(a.q, b.q, j);
			float clamped = phi < j.lowerAngle ? j.lowerAngle : (phi > j.upperAngle ? j.upperAngle : phi);
			if (clamped != phi)
			{
				V3 axis = rotate(a.q, j.localAxisA);
				applyAngularCorrection(a, b, scale(phi - clamped, axis));
			}
		}
	}
	else if (j.type == kJointWeld)
	{
		Q4 target = qmul(a.q, j.relRot0);
		Q4 qerr = qmul(b.q, qconj(target));
		float sign = qerr.w >= 0.0f ? 1.0f : -1.0f;
		applyAngularCorrection(a, b, scale(2.0f * sign, v3(qerr.x, qerr.y, qerr.z)));
	}

	V3 rA = rotate(a.q, j.localAnchorA);
	V3 rB = rotate(b.q, j.localAnchorB);
	V3 d = sub(add(b.p, rB), add(a.p, rA));
	float l = len(d);
	if (l >= 1e-9f)
	{
		V3 u = scale(1.0f / l, d);
		float Cc = j.type == kJointDistance ? l - j.length : l;
		float w = generalizedInvMass(a, rA, u) + generalizedInvMass(b, rB, u);
		float alphaTilde = j.compliance / (h * h);
		float denom = w + alphaTilde;
		if (denom > 0.0f)
		{
			float dLambda = (-Cc - alphaTilde * j.lambda) / denom;
			j.lambda += dLambda;
			V3 p = scale(dLambda, u);
			applyPositionCorrection(b, p, rB);
			applyPositionCorrection(a, neg(p), rA);
		}
	}
	storePose(B, j.bodyA, a);
	storePose(B, j.bodyB, b);
}

M3G_D void solveJointVelocity(const BodySoA& B, JointRec& j, float h)
{
	if (j.type != kJointHinge || !j.enableMotor || j.maxMotorTorque <= 0.0f)
	{
		return;
	}
	BodyDyn a = loadDyn(B, j.bodyA), b = loadDyn(B, j.bodyB);
	V3 axis = rotate(a.q, j.localAxisA);
	float wA = a.invMass != 0.0f ? dot(axis, mulv(a.iw, axis)) : 0.0f;
	float wB = b.invMass != 0.0f ? dot(axis, mulv(b.iw, axis)) : 0.0f;
	float denom = wA + wB;
	if (denom <= 0.0f)
	{
		return;
	}
	V3 wa = ld3(B.angVel[j.bodyA]), wb = ld3(B.angVel[j.bodyB]);
	float wrel = dot(sub(wb, wa), axis);
	float dLambda = (j.motorSpeed - wrel) / denom;
	float budget = j.maxMotorTorque * h;
	float nl = j.motorLambda + dLambda;
	nl = nl > budget ? budget : (nl < -budget ? -budget : nl);
	dLambda = nl - j.motorLambda;
	j.motorLambda = nl;
	V3 p = scale(dLambda, axis);
	if (b.invMass != 0.0f)
	{
		B.angVel[j.bodyB] = st3(add(wb, mulv(b.iw, p)));
	}
	if (a.invMass != 0.0f)
	{
		B.angVel[j.bodyA] = st3(sub(wa, mulv(a.iw, p)));
	}
}

// ---- shared by the island solve kernels ---------------------------------------

struct SolveParams
{
	float h, invH, maxCorrection, gravityLen;
	V3 gravity;
	int substeps;
	int iterations;
};

__device__ __forceinline__ void jointPosition(const BodySoA& B, JointRec* J, int ji, float h)
{
	JointRec jr = J[ji];
	solveJointPosition(B, jr, h);
	J[ji] = jr;
}
__device__ __forceinline__ void jointVelocity(const BodySoA& B, JointRec* J, int ji, float h)
{
	JointRec jr = J[ji];
	solveJointVelocity(B, jr, h);
	J[ji] = jr;
}
__device__ __forceinline__ void jointPrepare(const BodySoA& B, JointRec* J, int ji)
{
	JointRec jr = J[ji];
	prepareJoint(B, jr);
	J[ji] = jr;
}
__device__ __forceinline__ void jointReset(JointRec* J, int ji)
{
	J[ji].lambda = 0.0f;
	J[ji].motorLambda = 0.0f;
}

} // namespace m3g

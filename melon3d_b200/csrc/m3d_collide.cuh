// Narrowphase element routines: contact manifolds between sphere / capsule /
// box, friction-anchor inheritance, shape ray casts and shape AABBs.
//
// These are per-pair functions called by one GPU thread each (the
// narrowphase kernel, the per-substep safety re-collision and the tunnelling
// rescue).  They restate the reference's algorithms
// (src/collide.cpp, src/grid.cpp:145-174) operation for operation, because the
// manifold points feed a Gauss-Seidel solver whose results are compared with
// the reference bit for bit.
#pragma once

#include "m3d_types.cuh"

#include <float.h>

namespace m3g
{

// append one point; anchors are stored in each body's local frame
// (reference src/collide.cpp:16-34)
M3G_HD void pushPoint(Manifold* m, Xf xfA, Xf xfB, V3 onA, V3 onB, float sep, uint32_t id)
{
	if (m->pointCount >= 4)
	{
		return;
	}
	ManifoldPoint& p = m->points[m->pointCount++];
	p.localAnchorA = xfInvPoint(xfA, onA);
	p.localAnchorB = xfInvPoint(xfB, onB);
	p.frictionAnchorA = p.localAnchorA;
	p.frictionAnchorB = p.localAnchorB;
	p.separation = sep;
	p.id = id;
	p.lambdaN = 0.0f;
	p.lambdaT = 0.0f;
	p.separationOffset = 0.0f;
	p.slipDir = vzero();
}

// closest point to p on segment [a,b] (reference src/collide.cpp:36-47)
M3G_HD V3 closestOnSegment(V3 p, V3 a, V3 b)
{
	V3 ab = sub(b, a);
	float denom = dot(ab, ab);
	if (denom < 1e-12f)
	{
		return a;
	}
	float t = dot(sub(p, a), ab) / denom;
	t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
	return madd(a, t, ab);
}

// closest points between two segments, Ericson "Real-Time Collision
// Detection" 5.1.9 (reference src/collide.cpp:50-101)
M3G_HD void closestSegSeg(V3 p1, V3 q1, V3 p2, V3 q2, V3* c1, V3* c2)
{
	V3 d1 = sub(q1, p1);
	V3 d2 = sub(q2, p2);
	V3 r = sub(p1, p2);
	float a = dot(d1, d1);
	float e = dot(d2, d2);
	float f = dot(d2, r);
	float s, t;
	if (a < 1e-12f && e < 1e-12f)
	{
		*c1 = p1;
		*c2 = p2;
		return;
	}
	if (a < 1e-12f)
	{
		s = 0.0f;
		t = f / e;
	}
	else
	{
		float c = dot(d1, r);
		if (e < 1e-12f)
		{
			t = 0.0f;
			s = -c / a;
		}
		else
		{
			float b = dot(d1, d2);
			float denom = a * e - b * b;
			s = denom > 1e-12f ? (b * f - c * e) / denom : 0.0f;
			s = s < 0.0f ? 0.0f : (s > 1.0f ? 1.0f : s);
			t = (b * s + f) / e;
			if (t < 0.0f)
			{
				t = 0.0f;
				s = -c / a;
			}
			else if (t > 1.0f)
			{
				t = 1.0f;
				s = (b - c) / a;
			}
			s = s < 0.0f ? 0.0f : (s > 1.0f ? 1.0f : s);
		}
	}
	*c1 = madd(p1, s, d1);
	*c2 = madd(p2, t, d2);
}

M3G_HD V3 clampBox(V3 p, V3 e)
{
	V3 q;
	q.x = p.x < -e.x ? -e.x : (p.x > e.x ? e.x : p.x);
	q.y = p.y < -e.y ? -e.y : (p.y > e.y ? e.y : p.y);
	q.z = p.z < -e.z ? -e.z : (p.z > e.z ? e.z : p.z);
	return q;
}

// sphere-sphere (reference src/collide.cpp:116-130)
M3G_HD void collideSpheres(const Shape& a, Xf xfA, const Shape& b, Xf xfB, float margin, Manifold* m)
{
	V3 d = sub(xfB.p, xfA.p);
	float dist = len(d);
	V3 n = dist > 1e-9f ? scale(1.0f / dist, d) : v3(0.0f, 1.0f, 0.0f);
	float sep = dist - a.radius - b.radius;
	if (sep > margin)
	{
		return;
	}
	m->normal = n;
	pushPoint(m, xfA, xfB, madd(xfA.p, a.radius, n), madd(xfB.p, -b.radius, n), sep, 0);
}

// sphere (A) vs capsule (B) (reference src/collide.cpp:136-155)
M3G_HD void collideSphereCapsule(const Shape& a, Xf xfA, const Shape& b, Xf xfB, float margin, Manifold* m)
{
	V3 axis = rotate(xfB.q, v3(0.0f, b.halfHeight, 0.0f));
	V3 p1 = sub(xfB.p, axis);
	V3 p2 = add(xfB.p, axis);
	V3 c = closestOnSegment(xfA.p, p1, p2);
	V3 d = sub(c, xfA.p);
	float dist = len(d);
	V3 n = dist > 1e-9f ? scale(1.0f / dist, d) : v3(0.0f, 1.0f, 0.0f);
	float sep = dist - a.radius - b.radius;
	if (sep > margin)
	{
		return;
	}
	m->normal = n;
	pushPoint(m, xfA, xfB, madd(xfA.p, a.radius, n), madd(c, -b.radius, n), sep, 0);
}

// capsule vs capsule, with the two-point parallel case
// (reference src/collide.cpp:161-230)
M3G_HD void collideCapsules(const Shape& a, Xf xfA, const Shape& b, Xf xfB, float margin, Manifold* m)
{
	V3 axisA = rotate(xfA.q, v3(0.0f, a.halfHeight, 0.0f));
	V3 a1 = sub(xfA.p, axisA);
	V3 a2 = add(xfA.p, axisA);
	V3 axisB = rotate(xfB.q, v3(0.0f, b.halfHeight, 0.0f));
	V3 b1 = sub(xfB.p, axisB);
	V3 b2 = add(xfB.p, axisB);

	V3 uA = normalize(sub(a2, a1));
	V3 uB = normalize(sub(b2, b1));
	float parallelism = len(cross(uA, uB));

	if (parallelism < 0.05f && a.halfHeight > 1e-6f)
	{
		float lenA = 2.0f * a.halfHeight;
		float tb1 = dot(sub(b1, a1), uA);
		float tb2 = dot(sub(b2, a1), uA);
		float lo = fmaxf(0.0f, fminf(tb1, tb2));
		float hi = fminf(lenA, fmaxf(tb1, tb2));
		if (hi - lo > 1e-4f)
		{
			V3 midA = madd(a1, 0.5f * (lo + hi), uA);
			V3 midB = closestOnSegment(midA, b1, b2);
			V3 d = sub(midB, midA);
			float dist = len(d);
			V3 n = dist > 1e-9f ? scale(1.0f / dist, d) : v3(0.0f, 1.0f, 0.0f);
			if (dist - a.radius - b.radius > margin)
			{
				return;
			}
			m->normal = n;
			float ts[2] = { lo, hi };
			for (int i = 0; i < 2; ++i)
			{
				V3 cA = madd(a1, ts[i], uA);
				V3 cB = closestOnSegment(cA, b1, b2);
				float di = len(sub(cB, cA));
				float sep = di - a.radius - b.radius;
				if (sep <= margin)
				{
					pushPoint(m, xfA, xfB, madd(cA, a.radius, n), madd(cB, -b.radius, n), sep, (uint32_t)i);
				}
			}
			if (m->pointCount > 0)
			{
				return;
			}
		}
	}

	V3 cA, cB;
	closestSegSeg(a1, a2, b1, b2, &cA, &cB);
	V3 d = sub(cB, cA);
	float dist = len(d);
	V3 n = dist > 1e-9f ? scale(1.0f / dist, d) : v3(0.0f, 1.0f, 0.0f);
	float sep = dist - a.radius - b.radius;
	if (sep > margin)
	{
		return;
	}
	m->normal = n;
	pushPoint(m, xfA, xfB, madd(cA, a.radius, n), madd(cB, -b.radius, n), sep, 0);
}

// sphere (A) vs box (B) (reference src/collide.cpp:236-288)
M3G_HD void collideSphereBox(const Shape& a, Xf xfA, const Shape& b, Xf xfB, float margin, Manifold* m)
{
	V3 c = xfInvPoint(xfB, xfA.p);
	V3 e = b.he;
	V3 q = clampBox(c, e);
	V3 d = sub(c, q);
	float dist2 = len2(d);
	V3 nLocal;
	float sep;
	if (dist2 > 1e-12f)
	{
		float dist = sqrtf(dist2);
		nLocal = scale(1.0f / dist, d);
		sep = dist - a.radius;
	}
	else
	{
		float dx = e.x - fabsf(c.x);
		float dy = e.y - fabsf(c.y);
		float dz = e.z - fabsf(c.z);
		if (dx < dy && dx < dz)
		{
			nLocal = v3(c.x >= 0.0f ? 1.0f : -1.0f, 0.0f, 0.0f);
			sep = -(dx + a.radius);
			q = v3(nLocal.x * e.x, c.y, c.z);
		}
		else if (dy < dz)
		{
			nLocal = v3(0.0f, c.y >= 0.0f ? 1.0f : -1.0f, 0.0f);
			sep = -(dy + a.radius);
			q = v3(c.x, nLocal.y * e.y, c.z);
		}
		else
		{
			nLocal = v3(0.0f, 0.0f, c.z >= 0.0f ? 1.0f : -1.0f);
			sep = -(dz + a.radius);
			q = v3(c.x, c.y, nLocal.z * e.z);
		}
	}
	if (sep > margin)
	{
		return;
	}
	V3 nWorld = rotate(xfB.q, nLocal);
	m->normal = neg(nWorld);
	V3 pB = xfPoint(xfB, q);
	V3 pA = madd(xfA.p, a.radius, m->normal);
	pushPoint(m, xfA, xfB, pA, pB, sep, 0);
}

M3G_HD float pointBoxDist2(V3 p, V3 e)
{
	V3 q = clampBox(p, e);
	return len2(sub(p, q));
}

// capsule (A) vs box (B): ternary search along the core segment, deep case
// by least-penetration face, two points when lying parallel
// (reference src/collide.cpp:301-424)
M3G_HD void collideCapsuleBox(const Shape& a, Xf xfA, const Shape& b, Xf xfB, float margin, Manifold* m)
{
	V3 e = b.he;
	float r = a.radius;
	V3 axis = rotate(xfA.q, v3(0.0f, a.halfHeight, 0.0f));
	V3 segA = xfInvPoint(xfB, sub(xfA.p, axis));
	V3 segB = xfInvPoint(xfB, add(xfA.p, axis));
	V3 segDir = sub(segB, segA);

	float lo = 0.0f, hi = 1.0f;
	float segLen2 = len2(segDir);
	float tol = segLen2 > 1e-12f ? (kLinearSlop * kLinearSlop) / segLen2 : 1e-6f;
	for (int i = 0; i < 22; ++i)
	{
		if ((hi - lo) * (hi - lo) < tol)
		{
			break;
		}
		float t1 = lo + (hi - lo) / 3.0f;
		float t2 = hi - (hi - lo) / 3.0f;
		float d1 = pointBoxDist2(madd(segA, t1, segDir), e);
		float d2 = pointBoxDist2(madd(segA, t2, segDir), e);
		if (d1 < d2)
		{
			hi = t2;
		}
		else
		{
			lo = t1;
		}
	}
	float tStar = 0.5f * (lo + hi);
	V3 c = madd(segA, tStar, segDir);
	V3 q = clampBox(c, e);
	V3 diff = sub(c, q);
	float dist2 = len2(diff);

	V3 nLocal;
	float sep;
	bool deep = dist2 <= 1e-10f;
	if (!deep)
	{
		float dist = sqrtf(dist2);
		nLocal = scale(1.0f / dist, diff);
		sep = dist - r;
		if (sep > margin)
		{
			return;
		}
	}
	else
	{
		float dx = e.x - fabsf(c.x);
		float dy = e.y - fabsf(c.y);
		float dz = e.z - fabsf(c.z);
		if (dx < dy && dx < dz)
		{
			nLocal = v3(c.x >= 0.0f ? 1.0f : -1.0f, 0.0f, 0.0f);
			sep = -(dx + r);
		}
		else if (dy < dz)
		{
			nLocal = v3(0.0f, c.y >= 0.0f ? 1.0f : -1.0f, 0.0f);
			sep = -(dy + r);
		}
		else
		{
			nLocal = v3(0.0f, 0.0f, c.z >= 0.0f ? 1.0f : -1.0f);
			sep = -(dz + r);
		}
		q = sub(c, scale(sep + r, nLocal));
	}

	V3 nBoxToCap = rotate(xfB.q, nLocal);
	m->normal = neg(nBoxToCap);

	V3 u = normalize(segDir);
	if (fabsf(dot(u, nLocal)) < 0.05f && a.halfHeight > 1e-6f)
	{
		int added = 0;
		V3 ends[2] = { segA, segB };
		for (int i = 0; i < 2; ++i)
		{
			V3 p = ends[i];
			V3 qp = clampBox(p, e);
			V3 dp = sub(p, qp);
			float d2 = len2(dp);
			float s;
			if (d2 > 1e-10f)
			{
				s = sqrtf(d2) - r;
			}
			else
			{
				float extent = e.x * fabsf(nLocal.x) + e.y * fabsf(nLocal.y) + e.z * fabsf(nLocal.z);
				s = (dot(p, nLocal) - extent) - r;
				qp = sub(p, scale(dot(p, nLocal) - extent, nLocal));
			}
			if (s <= margin)
			{
				V3 pCap = madd(xfPoint(xfB, p), r, m->normal);
				V3 pBox = xfPoint(xfB, qp);
				pushPoint(m, xfA, xfB, pCap, pBox, s, (uint32_t)i);
				++added;
			}
		}
		if (added > 0)
		{
			return;
		}
	}

	V3 pCap = madd(xfPoint(xfB, c), r, m->normal);
	V3 pBox = xfPoint(xfB, q);
	pushPoint(m, xfA, xfB, pCap, pBox, sep, 4);
}

struct ClipVert
{
	V3 v;
	uint32_t id;
};

// Sutherland-Hodgman clip against dot(x, n) <= offset, at most 8 vertices out
// (reference src/collide.cpp:437-464)
M3G_HD int clipPoly(const ClipVert* in, int inCount, V3 n, float offset, uint32_t planeId, ClipVert* out)
{
	int outCount = 0;
	for (int i = 0; i < inCount; ++i)
	{
		const ClipVert v1 = in[i];
		const ClipVert v2 = in[(i + 1) % inCount];
		float d1 = dot(v1.v, n) - offset;
		float d2 = dot(v2.v, n) - offset;
		if (d1 <= 0.0f)
		{
			out[outCount++] = v1;
		}
		if (d1 * d2 < 0.0f && outCount < 8)
		{
			float t = d1 / (d1 - d2);
			out[outCount].v = lerp(v1.v, v2.v, t);
			out[outCount].id = ((v1.id ^ v2.id) << 8) | planeId;
			++outCount;
		}
		if (outCount >= 8)
		{
			break;
		}
	}
	return outCount;
}

// the edge of an OBB furthest along a world direction
// (reference src/collide.cpp:467-509)
M3G_HD void supportEdge(Xf xf, const M3& rot, V3 e, V3 dirWorld, V3* pOut, V3* qOut)
{
	V3 d = mulvT(rot, dirWorld);
	V3 ad = vabs(d);
	int edgeAxis = 0;
	if (ad.y < ad.x && ad.y <= ad.z)
	{
		edgeAxis = 1;
	}
	else if (ad.z < ad.x && ad.z <= ad.y)
	{
		edgeAxis = 2;
	}
	else if (ad.x <= ad.y && ad.x <= ad.z)
	{
		edgeAxis = 0;
	}
	float sx = d.x >= 0.0f ? 1.0f : -1.0f;
	float sy = d.y >= 0.0f ? 1.0f : -1.0f;
	float sz = d.z >= 0.0f ? 1.0f : -1.0f;
	V3 p = v3(sx * e.x, sy * e.y, sz * e.z);
	V3 q = p;
	if (edgeAxis == 0)
	{
		p.x = -e.x;
		q.x = e.x;
	}
	else if (edgeAxis == 1)
	{
		p.y = -e.y;
		q.y = e.y;
	}
	else
	{
		p.z = -e.z;
		q.z = e.z;
	}
	*pOut = xfPoint(xf, p);
	*qOut = xfPoint(xf, q);
}

M3G_HD float projRadius(const V3* axes, const float* ext, V3 n)
{
	return ext[0] * fabsf(dot(axes[0], n)) + ext[1] * fabsf(dot(axes[1], n)) + ext[2] * fabsf(dot(axes[2], n));
}

// box vs box: 15-axis SAT, face preference, edge-edge closest points or
// incident-face clipping reduced to 4 points (reference src/collide.cpp:511-805)
M3G_HD void collideBoxes(const Shape& a, Xf xfA, const Shape& b, Xf xfB, float margin, Manifold* m)
{
	M3 rotA = quatToMat(xfA.q);
	M3 rotB = quatToMat(xfB.q);
	V3 eA = a.he;
	V3 eB = b.he;
	V3 d = sub(xfB.p, xfA.p);

	const V3 axesA[3] = { rotA.cx, rotA.cy, rotA.cz };
	const V3 axesB[3] = { rotB.cx, rotB.cy, rotB.cz };
	const float extA[3] = { eA.x, eA.y, eA.z };
	const float extB[3] = { eB.x, eB.y, eB.z };

	float faceASep = -FLT_MAX;
	int faceAIndex = 0;
	for (int i = 0; i < 3; ++i)
	{
		float s = fabsf(dot(d, axesA[i])) - (extA[i] + projRadius(axesB, extB, axesA[i]));
		if (s > margin)
		{
			return;
		}
		if (s > faceASep)
		{
			faceASep = s;
			faceAIndex = i;
		}
	}
	float faceBSep = -FLT_MAX;
	int faceBIndex = 0;
	for (int i = 0; i < 3; ++i)
	{
		float s = fabsf(dot(d, axesB[i])) - (extB[i] + projRadius(axesA, extA, axesB[i]));
		if (s > margin)
		{
			return;
		}
		if (s > faceBSep)
		{
			faceBSep = s;
			faceBIndex = i;
		}
	}
	float edgeSep = -FLT_MAX;
	int edgeI = 0, edgeJ = 0;
	V3 edgeAxis = vzero();
	for (int i = 0; i < 3; ++i)
	{
		for (int j = 0; j < 3; ++j)
		{
			V3 axis = cross(axesA[i], axesB[j]);
			float l2 = len2(axis);
			if (l2 < 1e-8f)
			{
				continue;
			}
			axis = scale(1.0f / sqrtf(l2), axis);
			float s = fabsf(dot(d, axis)) - (projRadius(axesA, extA, axis) + projRadius(axesB, extB, axis));
			if (s > margin)
			{
				return;
			}
			if (s > edgeSep)
			{
				edgeSep = s;
				edgeI = i;
				edgeJ = j;
				edgeAxis = axis;
			}
		}
	}

	const float kRelTol = 0.95f;
	const float kAbsTol = 0.01f * kLinearSlop * 200.0f;
	float bestFaceSep = faceASep;
	bool refIsA = true;
	int refFace = faceAIndex;
	if (faceBSep > kRelTol * faceASep + kAbsTol)
	{
		bestFaceSep = faceBSep;
		refIsA = false;
		refFace = faceBIndex;
	}

	if (edgeSep > kRelTol * bestFaceSep + kAbsTol)
	{
		V3 n = edgeAxis;
		if (dot(d, n) < 0.0f)
		{
			n = neg(n);
		}
		V3 pA1, pA2, pB1, pB2;
		supportEdge(xfA, rotA, eA, n, &pA1, &pA2);
		supportEdge(xfB, rotB, eB, neg(n), &pB1, &pB2);
		V3 cA, cB;
		closestSegSeg(pA1, pA2, pB1, pB2, &cA, &cB);
		m->normal = n;
		pushPoint(m, xfA, xfB, cA, cB, edgeSep, 0xE0000000u | (uint32_t)(edgeI * 3 + edgeJ));
		return;
	}

	Xf xfRef = refIsA ? xfA : xfB;
	Xf xfInc = refIsA ? xfB : xfA;
	const M3 rotInc = refIsA ? rotB : rotA;
	const V3* refAxes = refIsA ? axesA : axesB;
	const V3* incAxes = refIsA ? axesB : axesA;
	const float* refExt = refIsA ? extA : extB;
	const float* incExt = refIsA ? extB : extA;
	V3 dRefToInc = refIsA ? d : neg(d);

	float refSign = dot(refAxes[refFace], dRefToInc) >= 0.0f ? 1.0f : -1.0f;
	V3 refNormal = scale(refSign, refAxes[refFace]);

	int incFace = 0;
	float minDot = FLT_MAX;
	float incSign = 1.0f;
	for (int i = 0; i < 3; ++i)
	{
		float dd = dot(incAxes[i], refNormal);
		if (dd < minDot)
		{
			minDot = dd;
			incFace = i;
			incSign = 1.0f;
		}
		if (-dd < minDot)
		{
			minDot = -dd;
			incFace = i;
			incSign = -1.0f;
		}
	}

	int iu = (incFace + 1) % 3;
	int iv = (incFace + 2) % 3;
	V3 incCenterLocal = vzero();
	setComp(incCenterLocal, incFace, incSign * incExt[incFace]);
	V3 uL = vzero(), vL = vzero();
	setComp(uL, iu, incExt[iu]);
	setComp(vL, iv, incExt[iv]);

	ClipVert poly[8], tmp[8];
	{
		V3 cW = xfPoint(xfInc, incCenterLocal);
		V3 uW = mulv(rotInc, uL);
		V3 vW = mulv(rotInc, vL);
		poly[0].v = add(add(cW, uW), vW);
		poly[0].id = 0;
		poly[1].v = add(sub(cW, uW), vW);
		poly[1].id = 1;
		poly[2].v = sub(sub(cW, uW), vW);
		poly[2].id = 2;
		poly[3].v = sub(add(cW, uW), vW);
		poly[3].id = 3;
	}
	int count = 4;

	int sideAxes[2] = { (refFace + 1) % 3, (refFace + 2) % 3 };
	for (int k = 0; k < 2; ++k)
	{
		int ax = sideAxes[k];
		V3 sn = refAxes[ax];
		float centerProj = dot(xfRef.p, sn);
		count = clipPoly(poly, count, sn, centerProj + refExt[ax], (uint32_t)(2 * k + 4), tmp);
		if (count == 0)
		{
			return;
		}
		count = clipPoly(tmp, count, neg(sn), -(centerProj - refExt[ax]), (uint32_t)(2 * k + 5), poly);
		if (count == 0)
		{
			return;
		}
	}

	float faceOffset = dot(xfRef.p, refNormal) + refExt[refFace];
	ClipVert kept[8];
	float seps[8];
	int keptCount = 0;
	for (int i = 0; i < count; ++i)
	{
		float s = dot(poly[i].v, refNormal) - faceOffset;
		if (s <= margin)
		{
			kept[keptCount] = poly[i];
			seps[keptCount] = s;
			++keptCount;
		}
	}
	if (keptCount == 0)
	{
		return;
	}

	int order[8];
	int reduced = 0;
	if (keptCount <= 4)
	{
		for (int i = 0; i < keptCount; ++i)
		{
			order[reduced++] = i;
		}
	}
	else
	{
		int i0 = 0;
		for (int i = 1; i < keptCount; ++i)
		{
			if (seps[i] < seps[i0])
			{
				i0 = i;
			}
		}
		int i1 = -1;
		float bestD = -1.0f;
		for (int i = 0; i < keptCount; ++i)
		{
			if (i == i0)
			{
				continue;
			}
			float dd = len2(sub(kept[i].v, kept[i0].v));
			if (dd > bestD)
			{
				bestD = dd;
				i1 = i;
			}
		}
		int i2 = -1, i3 = -1;
		float bestArea = 0.0f, worstArea = 0.0f;
		for (int i = 0; i < keptCount; ++i)
		{
			if (i == i0 || i == i1)
			{
				continue;
			}
			V3 e1 = sub(kept[i1].v, kept[i0].v);
			V3 e2 = sub(kept[i].v, kept[i0].v);
			float area = dot(cross(e1, e2), refNormal);
			if (area > bestArea)
			{
				bestArea = area;
				i2 = i;
			}
			if (area < worstArea)
			{
				worstArea = area;
				i3 = i;
			}
		}
		order[reduced++] = i0;
		order[reduced++] = i1;
		if (i2 >= 0)
		{
			order[reduced++] = i2;
		}
		if (i3 >= 0)
		{
			order[reduced++] = i3;
		}
	}

	m->normal = refIsA ? refNormal : neg(refNormal);
	uint32_t flipBit = refIsA ? 0u : 0x40000000u;
	for (int k = 0; k < reduced; ++k)
	{
		int i = order[k];
		V3 pInc = kept[i].v;
		V3 pRef = madd(pInc, -seps[i], refNormal);
		uint32_t id = (kept[i].id & 0x00FFFFFFu) | ((uint32_t)refFace << 24) | flipBit;
		if (refIsA)
		{
			pushPoint(m, xfA, xfB, pRef, pInc, seps[i], id);
		}
		else
		{
			pushPoint(m, xfA, xfB, pInc, pRef, seps[i], id);
		}
	}
}

// dispatch in canonical (type A <= type B) order; the flipped result swaps
// anchors and negates the normal (reference src/collide.cpp:813-859)
M3G_HD void collideCanonical(const Shape& a, Xf xfA, const Shape& b, Xf xfB, float margin, Manifold* m)
{
	m->pointCount = 0;
	m->normal = v3(0.0f, 1.0f, 0.0f);
	switch (a.type)
	{
		case kSphere:
			if (b.type == kSphere)
				collideSpheres(a, xfA, b, xfB, margin, m);
			else if (b.type == kCapsule)
				collideSphereCapsule(a, xfA, b, xfB, margin, m);
			else
				collideSphereBox(a, xfA, b, xfB, margin, m);
			return;
		case kCapsule:
			if (b.type == kCapsule)
				collideCapsules(a, xfA, b, xfB, margin, m);
			else if (b.type == kBox)
				collideCapsuleBox(a, xfA, b, xfB, margin, m);
			return;
		default:
			collideBoxes(a, xfA, b, xfB, margin, m);
			return;
	}
}

// Fresh manifold into *m.  Point slots at and beyond m->pointCount keep
// whatever they held before, exactly like the reference, which regenerates
// into the contact's existing manifold storage.
M3G_HD void collideShapes(const Shape& a, Xf xfA, const Shape& b, Xf xfB, float margin, Manifold* m)
{
	if (a.type > b.type)
	{
		Manifold f;
		collideCanonical(b, xfB, a, xfA, margin, &f);
		m->pointCount = f.pointCount;
		m->normal = neg(f.normal);
		for (int i = 0; i < f.pointCount; ++i)
		{
			ManifoldPoint p = f.points[i];
			V3 t = p.localAnchorA;
			p.localAnchorA = p.localAnchorB;
			p.localAnchorB = t;
			t = p.frictionAnchorA;
			p.frictionAnchorA = p.frictionAnchorB;
			p.frictionAnchorB = t;
			m->points[i] = p;
		}
		return;
	}
	collideCanonical(a, xfA, b, xfB, margin, m);
}

// Carry slip direction (all shapes) and, for box-box pairs that have not
// slipped, the stiction anchors from the previous manifold, matched by
// feature id (reference src/collide.cpp:865-913)
M3G_HD void inheritAnchors(const Manifold& old, Manifold& m, bool boxBox, Xf xfA, Xf xfB)
{
	const float kSlipReleaseSq = 0.02f * 0.02f;
	const float kFeatureDriftSq = 0.05f * 0.05f;
	V3 n = m.normal;
	for (int i = 0; i < m.pointCount; ++i)
	{
		ManifoldPoint& mp = m.points[i];
		for (int j = 0; j < old.pointCount; ++j)
		{
			const ManifoldPoint& op = old.points[j];
			if (op.id != mp.id)
			{
				continue;
			}
			mp.slipDir = op.slipDir;
			if (!boxBox)
			{
				break;
			}
			V3 pAold = add(xfA.p, rotate(xfA.q, op.frictionAnchorA));
			V3 pBold = add(xfB.p, rotate(xfB.q, op.frictionAnchorB));
			V3 pAnew = add(xfA.p, rotate(xfA.q, mp.localAnchorA));
			V3 gap = sub(pBold, pAold);
			V3 dpt = sub(gap, scale(dot(gap, n), n));
			if (len2(dpt) < kSlipReleaseSq && len2(sub(pAold, pAnew)) < kFeatureDriftSq)
			{
				mp.frictionAnchorA = op.frictionAnchorA;
				mp.frictionAnchorB = op.frictionAnchorB;
			}
			break;
		}
	}
}

// ---- ray casts (reference src/collide.cpp:919-1066) -----------------------

M3G_HD bool rayCastSphere(V3 center, float radius, V3 o, V3 d, float* fraction, V3* normal)
{
	V3 s = sub(o, center);
	float b = len2(s) - radius * radius;
	float rr = dot(s, d);
	float c = dot(d, d);
	float sigma = rr * rr - c * b;
	if (sigma < 0.0f || c < 1e-12f)
	{
		return false;
	}
	float t = -(rr + sqrtf(sigma)) / c;
	if (t < 0.0f || t > 1.0f)
	{
		return false;
	}
	*fraction = t;
	*normal = normalize(add(s, scale(t, d)));
	return true;
}

M3G_HD bool rayCastBoxLocal(V3 e, V3 o, V3 d, float* fraction, V3* normalLocal)
{
	float tmin = 0.0f, tmax = 1.0f;
	V3 n = vzero();
	for (int i = 0; i < 3; ++i)
	{
		float di = comp(d, i), oi = comp(o, i), ei = comp(e, i);
		if (fabsf(di) < 1e-12f)
		{
			if (oi < -ei || oi > ei)
			{
				return false;
			}
		}
		else
		{
			float inv = 1.0f / di;
			float t1 = (-ei - oi) * inv;
			float t2 = (ei - oi) * inv;
			float sign = -1.0f;
			if (t1 > t2)
			{
				float tt = t1;
				t1 = t2;
				t2 = tt;
				sign = 1.0f;
			}
			if (t1 > tmin)
			{
				tmin = t1;
				n = vzero();
				setComp(n, i, sign);
			}
			tmax = tmax < t2 ? tmax : t2;
			if (tmin > tmax)
			{
				return false;
			}
		}
	}
	if (len2(n) < 0.5f)
	{
		return false; // started inside
	}
	*fraction = tmin;
	*normalLocal = n;
	return true;
}

M3G_HD bool rayCastShape(const Shape& shape, Xf xf, V3 origin, V3 translation, float* fraction, V3* normal)
{
	switch (shape.type)
	{
		case kSphere:
			return rayCastSphere(xf.p, shape.radius, origin, translation, fraction, normal);
		case kBox:
		{
			V3 oL = xfInvPoint(xf, origin);
			V3 dL = invRotate(xf.q, translation);
			V3 nL;
			if (!rayCastBoxLocal(shape.he, oL, dL, fraction, &nL))
			{
				return false;
			}
			*normal = rotate(xf.q, nL);
			return true;
		}
		case kCapsule:
		{
			V3 oL = xfInvPoint(xf, origin);
			V3 dL = invRotate(xf.q, translation);
			float h = shape.halfHeight;
			float r = shape.radius;
			float best = FLT_MAX;
			V3 bestN = vzero();
			float aa = dL.x * dL.x + dL.z * dL.z;
			if (aa > 1e-12f)
			{
				float bb = oL.x * dL.x + oL.z * dL.z;
				float cc = oL.x * oL.x + oL.z * oL.z - r * r;
				float sigma = bb * bb - aa * cc;
				if (sigma >= 0.0f)
				{
					float t = (-bb - sqrtf(sigma)) / aa;
					if (t >= 0.0f && t <= 1.0f)
					{
						float y = oL.y + t * dL.y;
						if (fabsf(y) <= h)
						{
							best = t;
							V3 hp = madd(oL, t, dL);
							bestN = normalize(v3(hp.x, 0.0f, hp.z));
						}
					}
				}
			}
			for (int i = 0; i < 2; ++i)
			{
				V3 cap = v3(0.0f, i == 0 ? h : -h, 0.0f);
				float t;
				V3 n;
				if (rayCastSphere(cap, r, oL, dL, &t, &n) && t < best)
				{
					best = t;
					bestN = n;
				}
			}
			if (best == FLT_MAX)
			{
				return false;
			}
			*fraction = best;
			*normal = rotate(xf.q, bestN);
			return true;
		}
	}
	return false;
}

// tight shape AABB (reference src/grid.cpp:145-174)
M3G_HD Box shapeAABB(const Shape& s, Xf xf)
{
	Box b;
	switch (s.type)
	{
		case kSphere:
		{
			V3 r = v3(s.radius, s.radius, s.radius);
			b.lo = sub(xf.p, r);
			b.hi = add(xf.p, r);
			return b;
		}
		case kCapsule:
		{
			V3 axis = rotate(xf.q, v3(0.0f, s.halfHeight, 0.0f));
			V3 p1 = add(xf.p, axis);
			V3 p2 = sub(xf.p, axis);
			V3 r = v3(s.radius, s.radius, s.radius);
			b.lo = sub(vmin(p1, p2), r);
			b.hi = add(vmax(p1, p2), r);
			return b;
		}
		default:
		{
			M3 rot = quatToMat(xf.q);
			V3 e = s.he;
			V3 ext;
			ext.x = fabsf(rot.cx.x) * e.x + fabsf(rot.cy.x) * e.y + fabsf(rot.cz.x) * e.z;
			ext.y = fabsf(rot.cx.y) * e.x + fabsf(rot.cy.y) * e.y + fabsf(rot.cz.y) * e.z;
			ext.z = fabsf(rot.cx.z) * e.x + fabsf(rot.cy.z) * e.y + fabsf(rot.cz.z) * e.z;
			b.lo = sub(xf.p, ext);
			b.hi = add(xf.p, ext);
			return b;
		}
	}
}

} // namespace m3g

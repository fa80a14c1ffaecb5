// Differentiable manifold generation: the engine's narrowphase for spheres
// and boxes (m3d_collide.cuh; reference src/collide.cpp:116-130, 236-288,
// 511-859) restated over a generic scalar, evaluated with forward-mode dual
// numbers to get the derivatives of a generated manifold (normal, local
// anchors, separation offsets) with respect to the two poses it was
// generated at.
//
// With S = Dual<float, N> the value parts repeat the engine's float
// operations in the engine's order, so every branch (SAT axis, reference
// face, clipping, the sep <= margin test, the reduction to four points)
// falls the way it fell in the engine and the derivatives are those of the
// branch the engine took.  With S = Dual<double, N> (the FP64 host reference)
// a branch can differ on a near tie; points are then matched by feature id and
// an unmatched point contributes nothing.  With S = float or double (no
// derivatives) it is the manifold regeneration of the regenerating replay.
//
// Included by m3d_diff.h.
#pragma once

#include <float.h>

namespace m3d_diff
{

// ---- dual numbers -------------------------------------------------------------

// value in T (float: the engine's own rounding, so its branches), derivatives
// in double (a generation's derivative terms cancel strongly)
template <typename T, int N>
struct Dual
{
	T v;
	double d[N];
	M3D_DIFF_HD Dual() : v(T(0))
	{
		for (int i = 0; i < N; ++i)
			d[i] = 0.0;
	}
	M3D_DIFF_HD Dual(T x) : v(x)
	{
		for (int i = 0; i < N; ++i)
			d[i] = 0.0;
	}
};

template <typename T, int N>
M3D_DIFF_HD Dual<T, N> operator+(const Dual<T, N>& a, const Dual<T, N>& b)
{
	Dual<T, N> r;
	r.v = a.v + b.v;
	for (int i = 0; i < N; ++i)
		r.d[i] = a.d[i] + b.d[i];
	return r;
}
template <typename T, int N>
M3D_DIFF_HD Dual<T, N> operator-(const Dual<T, N>& a, const Dual<T, N>& b)
{
	Dual<T, N> r;
	r.v = a.v - b.v;
	for (int i = 0; i < N; ++i)
		r.d[i] = a.d[i] - b.d[i];
	return r;
}
template <typename T, int N>
M3D_DIFF_HD Dual<T, N> operator-(const Dual<T, N>& a)
{
	Dual<T, N> r;
	r.v = -a.v;
	for (int i = 0; i < N; ++i)
		r.d[i] = -a.d[i];
	return r;
}
template <typename T, int N>
M3D_DIFF_HD Dual<T, N> operator*(const Dual<T, N>& a, const Dual<T, N>& b)
{
	Dual<T, N> r;
	r.v = a.v * b.v;
	for (int i = 0; i < N; ++i)
		r.d[i] = a.d[i] * (double)b.v + (double)a.v * b.d[i];
	return r;
}
template <typename T, int N>
M3D_DIFF_HD Dual<T, N> operator/(const Dual<T, N>& a, const Dual<T, N>& b)
{
	Dual<T, N> r;
	r.v = a.v / b.v;
	const double q = (double)a.v / (double)b.v, ib = 1.0 / (double)b.v;
	for (int i = 0; i < N; ++i)
		r.d[i] = (a.d[i] - q * b.d[i]) * ib;
	return r;
}
template <typename T, int N>
M3D_DIFF_HD bool operator<(const Dual<T, N>& a, const Dual<T, N>& b)
{
	return a.v < b.v;
}
template <typename T, int N>
M3D_DIFF_HD bool operator>(const Dual<T, N>& a, const Dual<T, N>& b)
{
	return a.v > b.v;
}
template <typename T, int N>
M3D_DIFF_HD bool operator<=(const Dual<T, N>& a, const Dual<T, N>& b)
{
	return a.v <= b.v;
}
template <typename T, int N>
M3D_DIFF_HD bool operator>=(const Dual<T, N>& a, const Dual<T, N>& b)
{
	return a.v >= b.v;
}
template <typename T, int N>
M3D_DIFF_HD Dual<T, N> dsqrt(const Dual<T, N>& a)
{
	Dual<T, N> r;
	r.v = dsqrt(a.v);
	const double k = r.v > T(0) ? 0.5 / dsqrt((double)a.v) : 0.0;
	for (int i = 0; i < N; ++i)
		r.d[i] = k * a.d[i];
	return r;
}
template <typename T, int N>
M3D_DIFF_HD Dual<T, N> dabs(const Dual<T, N>& a)
{
	return a.v < T(0) ? -a : a;
}

// ---- generated manifold ---------------------------------------------------------

template <typename S>
struct GenPoint
{
	V<S> la, lb;
	S sep, off;
	uint32_t id;
};
template <typename S>
struct GenManifold
{
	V<S> n;
	int count;
	GenPoint<S> p[4];
};

// engine constants used by the generation (reference src/m3d_internal.h:32-63)
constexpr float kGenLinearSlop = 0.005f;
constexpr float kGenSpeculativeBase = 4.0f * kGenLinearSlop;

template <typename S>
M3D_DIFF_HD V<S> gLerp(V<S> a, V<S> b, S t)
{
	return add(a, scale(t, sub(b, a)));
}
template <typename S>
M3D_DIFF_HD V<S> gXfPoint(V<S> x, Q<S> q, V<S> p)
{
	return add(rotate(q, p), x);
}
template <typename S>
M3D_DIFF_HD V<S> gXfInvPoint(V<S> x, Q<S> q, V<S> p)
{
	return rotate(qconj(q), sub(p, x));
}
template <typename S>
M3D_DIFF_HD M<S> gQuatToMat(Q<S> q)
{
	S x = q.x, y = q.y, z = q.z, w = q.w;
	S x2 = x + x, y2 = y + y, z2 = z + z;
	S xx = x * x2, xy = x * y2, xz = x * z2;
	S yy = y * y2, yz = y * z2, zz = z * z2;
	S wx = w * x2, wy = w * y2, wz = w * z2;
	M<S> m;
	m.cx = v3<S>(S(1.0f) - (yy + zz), xy + wz, xz - wy);
	m.cy = v3<S>(xy - wz, S(1.0f) - (xx + zz), yz + wx);
	m.cz = v3<S>(xz + wy, yz - wx, S(1.0f) - (xx + yy));
	return m;
}
template <typename S>
M3D_DIFF_HD V<S> gMulvT(const M<S>& m, V<S> v)
{
	return v3<S>(dot(m.cx, v), dot(m.cy, v), dot(m.cz, v));
}
template <typename S>
M3D_DIFF_HD void gSetComp(V<S>& v, int i, S f)
{
	if (i == 0)
		v.x = f;
	else if (i == 1)
		v.y = f;
	else
		v.z = f;
}

template <typename S>
M3D_DIFF_HD void gPush(GenManifold<S>& m, V<S> xA, Q<S> qA, V<S> xB, Q<S> qB, V<S> onA, V<S> onB, S sep, uint32_t id)
{
	if (m.count >= 4)
	{
		return;
	}
	GenPoint<S>& p = m.p[m.count++];
	p.la = gXfInvPoint(xA, qA, onA);
	p.lb = gXfInvPoint(xB, qB, onB);
	p.sep = sep;
	p.off = S(0.0f);
	p.id = id;
}

template <typename S>
M3D_DIFF_HD void gSpheres(S ra, V<S> xA, Q<S> qA, S rb, V<S> xB, Q<S> qB, S margin, GenManifold<S>& m)
{
	V<S> d = sub(xB, xA);
	S dist = len(d);
	V<S> n = dist > S(1e-9f) ? scale(S(1.0f) / dist, d) : v3<S>(S(0.0f), S(1.0f), S(0.0f));
	S sep = dist - ra - rb;
	if (sep > margin)
	{
		return;
	}
	m.n = n;
	gPush(m, xA, qA, xB, qB, madd(xA, ra, n), madd(xB, -rb, n), sep, 0u);
}

template <typename S>
M3D_DIFF_HD V<S> gClampBox(V<S> p, V<S> e)
{
	V<S> q;
	q.x = p.x < -e.x ? -e.x : (p.x > e.x ? e.x : p.x);
	q.y = p.y < -e.y ? -e.y : (p.y > e.y ? e.y : p.y);
	q.z = p.z < -e.z ? -e.z : (p.z > e.z ? e.z : p.z);
	return q;
}

template <typename S>
M3D_DIFF_HD_CALL void gSphereBox(S ra, V<S> xA, Q<S> qA, V<S> e, V<S> xB, Q<S> qB, S margin, GenManifold<S>& m)
{
	V<S> c = gXfInvPoint(xB, qB, xA);
	V<S> q = gClampBox(c, e);
	V<S> d = sub(c, q);
	S dist2 = dot(d, d);
	V<S> nLocal;
	S sep;
	if (dist2 > S(1e-12f))
	{
		S dist = dsqrt(dist2);
		nLocal = scale(S(1.0f) / dist, d);
		sep = dist - ra;
	}
	else
	{
		S dx = e.x - dabs(c.x);
		S dy = e.y - dabs(c.y);
		S dz = e.z - dabs(c.z);
		if (dx < dy && dx < dz)
		{
			nLocal = v3<S>(c.x >= S(0.0f) ? S(1.0f) : S(-1.0f), S(0.0f), S(0.0f));
			sep = -(dx + ra);
			q = v3<S>(nLocal.x * e.x, c.y, c.z);
		}
		else if (dy < dz)
		{
			nLocal = v3<S>(S(0.0f), c.y >= S(0.0f) ? S(1.0f) : S(-1.0f), S(0.0f));
			sep = -(dy + ra);
			q = v3<S>(c.x, nLocal.y * e.y, c.z);
		}
		else
		{
			nLocal = v3<S>(S(0.0f), S(0.0f), c.z >= S(0.0f) ? S(1.0f) : S(-1.0f));
			sep = -(dz + ra);
			q = v3<S>(c.x, c.y, nLocal.z * e.z);
		}
	}
	if (sep > margin)
	{
		return;
	}
	V<S> nWorld = rotate(qB, nLocal);
	m.n = neg(nWorld);
	V<S> pB = gXfPoint(xB, qB, q);
	V<S> pA = madd(xA, ra, m.n);
	gPush(m, xA, qA, xB, qB, pA, pB, sep, 0u);
}

template <typename S>
struct GClip
{
	V<S> v;
	uint32_t id;
};

template <typename S>
M3D_DIFF_HD_CALL int gClipPoly(const GClip<S>* in, int inCount, V<S> n, S offset, uint32_t planeId, GClip<S>* out)
{
	int outCount = 0;
	for (int i = 0; i < inCount; ++i)
	{
		const GClip<S> v1 = in[i];
		const GClip<S> v2 = in[(i + 1) % inCount];
		S d1 = dot(v1.v, n) - offset;
		S d2 = dot(v2.v, n) - offset;
		if (d1 <= S(0.0f))
		{
			out[outCount++] = v1;
		}
		if (d1 * d2 < S(0.0f) && outCount < 8)
		{
			S t = d1 / (d1 - d2);
			out[outCount].v = gLerp(v1.v, v2.v, t);
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

template <typename S>
M3D_DIFF_HD_CALL void gSupportEdge(V<S> x, Q<S> qq, const M<S>& rot, V<S> e, V<S> dirWorld, V<S>* pOut, V<S>* qOut)
{
	V<S> d = gMulvT(rot, dirWorld);
	V<S> ad = v3<S>(dabs(d.x), dabs(d.y), dabs(d.z));
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
	S sx = d.x >= S(0.0f) ? S(1.0f) : S(-1.0f);
	S sy = d.y >= S(0.0f) ? S(1.0f) : S(-1.0f);
	S sz = d.z >= S(0.0f) ? S(1.0f) : S(-1.0f);
	V<S> p = v3<S>(sx * e.x, sy * e.y, sz * e.z);
	V<S> q = p;
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
	*pOut = gXfPoint(x, qq, p);
	*qOut = gXfPoint(x, qq, q);
}

template <typename S>
M3D_DIFF_HD S gProjRadius(const V<S>* axes, const S* ext, V<S> n)
{
	return ext[0] * dabs(dot(axes[0], n)) + ext[1] * dabs(dot(axes[1], n)) + ext[2] * dabs(dot(axes[2], n));
}

template <typename S>
M3D_DIFF_HD_CALL void gClosestSegSeg(V<S> p1, V<S> q1, V<S> p2, V<S> q2, V<S>* c1, V<S>* c2)
{
	V<S> d1 = sub(q1, p1);
	V<S> d2 = sub(q2, p2);
	V<S> r = sub(p1, p2);
	S a = dot(d1, d1);
	S e = dot(d2, d2);
	S f = dot(d2, r);
	S s, t;
	if (a < S(1e-12f) && e < S(1e-12f))
	{
		*c1 = p1;
		*c2 = p2;
		return;
	}
	if (a < S(1e-12f))
	{
		s = S(0.0f);
		t = f / e;
	}
	else
	{
		S c = dot(d1, r);
		if (e < S(1e-12f))
		{
			t = S(0.0f);
			s = -c / a;
		}
		else
		{
			S b = dot(d1, d2);
			S denom = a * e - b * b;
			s = denom > S(1e-12f) ? (b * f - c * e) / denom : S(0.0f);
			s = s < S(0.0f) ? S(0.0f) : (s > S(1.0f) ? S(1.0f) : s);
			t = (b * s + f) / e;
			if (t < S(0.0f))
			{
				t = S(0.0f);
				s = -c / a;
			}
			else if (t > S(1.0f))
			{
				t = S(1.0f);
				s = (b - c) / a;
			}
			s = s < S(0.0f) ? S(0.0f) : (s > S(1.0f) ? S(1.0f) : s);
		}
	}
	*c1 = madd(p1, s, d1);
	*c2 = madd(p2, t, d2);
}

template <typename S>
M3D_DIFF_HD_CALL void gBoxes(V<S> eA, V<S> xA, Q<S> qA, V<S> eB, V<S> xB, Q<S> qB, S margin, GenManifold<S>& m)
{
	M<S> rotA = gQuatToMat(qA);
	M<S> rotB = gQuatToMat(qB);
	V<S> d = sub(xB, xA);
	const V<S> axesA[3] = { rotA.cx, rotA.cy, rotA.cz };
	const V<S> axesB[3] = { rotB.cx, rotB.cy, rotB.cz };
	const S extA[3] = { eA.x, eA.y, eA.z };
	const S extB[3] = { eB.x, eB.y, eB.z };

	S faceASep = S(-FLT_MAX);
	int faceAIndex = 0;
	for (int i = 0; i < 3; ++i)
	{
		S s = dabs(dot(d, axesA[i])) - (extA[i] + gProjRadius(axesB, extB, axesA[i]));
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
	S faceBSep = S(-FLT_MAX);
	int faceBIndex = 0;
	for (int i = 0; i < 3; ++i)
	{
		S s = dabs(dot(d, axesB[i])) - (extB[i] + gProjRadius(axesA, extA, axesB[i]));
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
	S edgeSep = S(-FLT_MAX);
	int edgeI = 0, edgeJ = 0;
	V<S> edgeAxis = vzero<S>();
	for (int i = 0; i < 3; ++i)
	{
		for (int j = 0; j < 3; ++j)
		{
			V<S> axis = cross(axesA[i], axesB[j]);
			S l2 = dot(axis, axis);
			if (l2 < S(1e-8f))
			{
				continue;
			}
			axis = scale(S(1.0f) / dsqrt(l2), axis);
			S s = dabs(dot(d, axis)) - (gProjRadius(axesA, extA, axis) + gProjRadius(axesB, extB, axis));
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

	const S kRelTol = S(0.95f);
	const S kAbsTol = S(0.01f * kGenLinearSlop * 200.0f);
	S bestFaceSep = faceASep;
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
		V<S> n = edgeAxis;
		if (dot(d, n) < S(0.0f))
		{
			n = neg(n);
		}
		V<S> pA1, pA2, pB1, pB2;
		gSupportEdge(xA, qA, rotA, eA, n, &pA1, &pA2);
		gSupportEdge(xB, qB, rotB, eB, neg(n), &pB1, &pB2);
		V<S> cA, cB;
		gClosestSegSeg(pA1, pA2, pB1, pB2, &cA, &cB);
		m.n = n;
		gPush(m, xA, qA, xB, qB, cA, cB, edgeSep, 0xE0000000u | (uint32_t)(edgeI * 3 + edgeJ));
		return;
	}

	V<S> xRef = refIsA ? xA : xB;
	V<S> xInc = refIsA ? xB : xA;
	Q<S> qInc = refIsA ? qB : qA;
	const M<S> rotInc = refIsA ? rotB : rotA;
	const V<S>* refAxes = refIsA ? axesA : axesB;
	const V<S>* incAxes = refIsA ? axesB : axesA;
	const S* refExt = refIsA ? extA : extB;
	const S* incExt = refIsA ? extB : extA;
	V<S> dRefToInc = refIsA ? d : neg(d);

	S refSign = dot(refAxes[refFace], dRefToInc) >= S(0.0f) ? S(1.0f) : S(-1.0f);
	V<S> refNormal = scale(refSign, refAxes[refFace]);

	int incFace = 0;
	S minDot = S(FLT_MAX);
	S incSign = S(1.0f);
	for (int i = 0; i < 3; ++i)
	{
		S dd = dot(incAxes[i], refNormal);
		if (dd < minDot)
		{
			minDot = dd;
			incFace = i;
			incSign = S(1.0f);
		}
		if (-dd < minDot)
		{
			minDot = -dd;
			incFace = i;
			incSign = S(-1.0f);
		}
	}

	int iu = (incFace + 1) % 3;
	int iv = (incFace + 2) % 3;
	V<S> incCenterLocal = vzero<S>();
	gSetComp(incCenterLocal, incFace, incSign * incExt[incFace]);
	V<S> uL = vzero<S>(), vL = vzero<S>();
	gSetComp(uL, iu, incExt[iu]);
	gSetComp(vL, iv, incExt[iv]);

	GClip<S> poly[8], tmp[8];
	{
		V<S> cW = gXfPoint(xInc, qInc, incCenterLocal);
		V<S> uW = mulv(rotInc, uL);
		V<S> vW = mulv(rotInc, vL);
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
		V<S> sn = refAxes[ax];
		S centerProj = dot(xRef, sn);
		count = gClipPoly(poly, count, sn, centerProj + refExt[ax], (uint32_t)(2 * k + 4), tmp);
		if (count == 0)
		{
			return;
		}
		count = gClipPoly(tmp, count, neg(sn), -(centerProj - refExt[ax]), (uint32_t)(2 * k + 5), poly);
		if (count == 0)
		{
			return;
		}
	}

	S faceOffset = dot(xRef, refNormal) + refExt[refFace];
	GClip<S> kept[8];
	S seps[8];
	int keptCount = 0;
	for (int i = 0; i < count; ++i)
	{
		S s = dot(poly[i].v, refNormal) - faceOffset;
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
		S bestD = S(-1.0f);
		for (int i = 0; i < keptCount; ++i)
		{
			if (i == i0)
			{
				continue;
			}
			V<S> dv = sub(kept[i].v, kept[i0].v);
			S dd = dot(dv, dv);
			if (dd > bestD)
			{
				bestD = dd;
				i1 = i;
			}
		}
		int i2 = -1, i3 = -1;
		S bestArea = S(0.0f), worstArea = S(0.0f);
		for (int i = 0; i < keptCount; ++i)
		{
			if (i == i0 || i == i1)
			{
				continue;
			}
			V<S> e1 = sub(kept[i1].v, kept[i0].v);
			V<S> e2 = sub(kept[i].v, kept[i0].v);
			S area = dot(cross(e1, e2), refNormal);
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

	m.n = refIsA ? refNormal : neg(refNormal);
	uint32_t flipBit = refIsA ? 0u : 0x40000000u;
	for (int k = 0; k < reduced; ++k)
	{
		int i = order[k];
		V<S> pInc = kept[i].v;
		V<S> pRef = madd(pInc, -seps[i], refNormal);
		uint32_t id = (kept[i].id & 0x00FFFFFFu) | ((uint32_t)refFace << 24) | flipBit;
		if (refIsA)
		{
			gPush(m, xA, qA, xB, qB, pRef, pInc, seps[i], id);
		}
		else
		{
			gPush(m, xA, qA, xB, qB, pInc, pRef, seps[i], id);
		}
	}
}

// one shape of a generation: type, sphere radius, box half extents
template <typename S>
struct GenShape
{
	int type;
	S radius;
	V<S> he;
};

template <typename S>
M3D_DIFF_HD void gCanonical(const GenShape<S>& a, V<S> xA, Q<S> qA, const GenShape<S>& b, V<S> xB, Q<S> qB, S margin,
							GenManifold<S>& m)
{
	m.count = 0;
	m.n = v3<S>(S(0.0f), S(1.0f), S(0.0f));
	if (a.type == kShapeSphere)
	{
		if (b.type == kShapeSphere)
			gSpheres(a.radius, xA, qA, b.radius, xB, qB, margin, m);
		else
			gSphereBox(a.radius, xA, qA, b.he, xB, qB, margin, m);
		return;
	}
	gBoxes(a.he, xA, qA, b.he, xB, qB, margin, m);
}

// A fresh manifold between body A and body B (contact order), with the
// separation offsets the engine stores: sep - n.(pB + rB - pA - rA) at the
// generation pose (reference src/world.cpp:1738-1845).
template <typename S>
M3D_DIFF_HD void genManifold(const GenShape<S>& a, V<S> xA, Q<S> qA, const GenShape<S>& b, V<S> xB, Q<S> qB,
							 S margin, GenManifold<S>& m)
{
	if (a.type > b.type)
	{
		GenManifold<S> f;
		gCanonical(b, xB, qB, a, xA, qA, margin, f);
		m.count = f.count;
		m.n = neg(f.n);
		for (int i = 0; i < f.count; ++i)
		{
			m.p[i] = f.p[i];
			m.p[i].la = f.p[i].lb;
			m.p[i].lb = f.p[i].la;
		}
	}
	else
	{
		gCanonical(a, xA, qA, b, xB, qB, margin, m);
	}
	for (int i = 0; i < m.count; ++i)
	{
		V<S> rA = rotate(qA, m.p[i].la);
		V<S> rB = rotate(qB, m.p[i].lb);
		S ref = dot(sub(add(xB, rB), add(xA, rA)), m.n);
		m.p[i].off = m.p[i].sep - ref;
	}
}

} // namespace m3d_diff

// Vector / quaternion arithmetic shared by every kernel.
//
// Parity rule: each helper performs the same float operations, in the same
// order, as the public inline math of include/melon3d.h (reference
// include/melon3d.h:85-233).  The library is compiled with --fmad=false and
// IEEE division/sqrt, so a kernel that composes these helpers the way the
// reference composes its own rounds bit-for-bit like the reference built with
// contraction off.  Nothing here may be "simplified" (dropping a 0*x term,
// reassociating a sum, replacing a division by a reciprocal multiply).
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define M3G_HD __host__ __device__ __forceinline__
#define M3G_D __device__ __forceinline__
#else
#define M3G_HD inline
#define M3G_D inline
#endif

namespace m3g
{

struct V3
{
	float x, y, z;
};
struct Q4
{
	float x, y, z, w;
};
struct M3
{
	V3 cx, cy, cz;
};
struct Xf
{
	V3 p;
	Q4 q;
};
struct Box
{
	V3 lo, hi;
};

M3G_HD V3 v3(float x, float y, float z)
{
	V3 r;
	r.x = x;
	r.y = y;
	r.z = z;
	return r;
}
M3G_HD V3 vzero() { return v3(0.0f, 0.0f, 0.0f); }
M3G_HD Q4 q4(float x, float y, float z, float w)
{
	Q4 r;
	r.x = x;
	r.y = y;
	r.z = z;
	r.w = w;
	return r;
}
M3G_HD Q4 qid() { return q4(0.0f, 0.0f, 0.0f, 1.0f); }

M3G_HD V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
M3G_HD V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
M3G_HD V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
M3G_HD V3 scale(float s, V3 v) { return v3(s * v.x, s * v.y, s * v.z); }
// a + s*b, component-wise
M3G_HD V3 madd(V3 a, float s, V3 b) { return v3(a.x + s * b.x, a.y + s * b.y, a.z + s * b.z); }
M3G_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
M3G_HD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
M3G_HD float len2(V3 v) { return dot(v, v); }
M3G_HD float len(V3 v) { return sqrtf(dot(v, v)); }
M3G_HD V3 normalize(V3 v)
{
	float l = len(v);
	if (l < 1e-12f)
	{
		return vzero();
	}
	float inv = 1.0f / l;
	return scale(inv, v);
}
M3G_HD V3 vmin(V3 a, V3 b) { return v3(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z); }
M3G_HD V3 vmax(V3 a, V3 b) { return v3(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z); }
M3G_HD V3 vabs(V3 a) { return v3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
M3G_HD V3 lerp(V3 a, V3 b, float t) { return add(a, scale(t, sub(b, a))); }
M3G_HD float comp(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
M3G_HD void setComp(V3& v, int i, float f)
{
	if (i == 0)
		v.x = f;
	else if (i == 1)
		v.y = f;
	else
		v.z = f;
}

M3G_HD Q4 qmul(Q4 a, Q4 b)
{
	Q4 q;
	q.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
	q.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
	q.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
	q.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
	return q;
}
M3G_HD Q4 qnormalize(Q4 q)
{
	float l = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
	if (l < 1e-12f)
	{
		return qid();
	}
	float inv = 1.0f / l;
	return q4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
}
M3G_HD Q4 qconj(Q4 q) { return q4(-q.x, -q.y, -q.z, q.w); }
// v + w*t + u x t, t = 2 u x v
M3G_HD V3 rotate(Q4 q, V3 v)
{
	V3 u = v3(q.x, q.y, q.z);
	V3 t = scale(2.0f, cross(u, v));
	return add(add(v, scale(q.w, t)), cross(u, t));
}
M3G_HD V3 invRotate(Q4 q, V3 v) { return rotate(qconj(q), v); }
M3G_HD Q4 qintegrate(Q4 q, V3 w, float h)
{
	Q4 wq = q4(w.x, w.y, w.z, 0.0f);
	Q4 dq = qmul(wq, q);
	Q4 r = q4(q.x + 0.5f * h * dq.x, q.y + 0.5f * h * dq.y, q.z + 0.5f * h * dq.z, q.w + 0.5f * h * dq.w);
	return qnormalize(r);
}
// first-order renormalisation q * (1.5 - 0.5 |q|^2) (reference src/xpbd.cpp:21-25)
M3G_HD Q4 qrenormFast(Q4 q)
{
	float s = 1.5f - 0.5f * (q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
	return q4(q.x * s, q.y * s, q.z * s, q.w * s);
}
M3G_HD M3 quatToMat(Q4 q)
{
	float x = q.x, y = q.y, z = q.z, w = q.w;
	float x2 = x + x, y2 = y + y, z2 = z + z;
	float xx = x * x2, xy = x * y2, xz = x * z2;
	float yy = y * y2, yz = y * z2, zz = z * z2;
	float wx = w * x2, wy = w * y2, wz = w * z2;
	M3 m;
	m.cx = v3(1.0f - (yy + zz), xy + wz, xz - wy);
	m.cy = v3(xy - wz, 1.0f - (xx + zz), yz + wx);
	m.cz = v3(xz + wy, yz - wx, 1.0f - (xx + yy));
	return m;
}
M3G_HD V3 mulv(const M3& m, V3 v) { return add(add(scale(v.x, m.cx), scale(v.y, m.cy)), scale(v.z, m.cz)); }
M3G_HD V3 mulvT(const M3& m, V3 v) { return v3(dot(m.cx, v), dot(m.cy, v), dot(m.cz, v)); }
M3G_HD V3 xfPoint(Xf xf, V3 p) { return add(rotate(xf.q, p), xf.p); }
M3G_HD V3 xfInvPoint(Xf xf, V3 p) { return invRotate(xf.q, sub(p, xf.p)); }
M3G_HD bool overlap(Box a, Box b)
{
	return a.lo.x <= b.hi.x && a.lo.y <= b.hi.y && a.lo.z <= b.hi.z && b.lo.x <= a.hi.x && b.lo.y <= a.hi.y &&
		   b.lo.z <= a.hi.z;
}
M3G_HD bool contains(Box a, Box b)
{
	return a.lo.x <= b.lo.x && a.lo.y <= b.lo.y && a.lo.z <= b.lo.z && b.hi.x <= a.hi.x && b.hi.y <= a.hi.y &&
		   b.hi.z <= a.hi.z;
}

// I^-1_world = R diag(d) R^T with the element order of the reference
// (src/m3d_internal.h:126-146)
M3G_HD M3 invInertiaWorld(Q4 rot, V3 d)
{
	M3 r = quatToMat(rot);
	M3 rd;
	rd.cx = scale(d.x, r.cx);
	rd.cy = scale(d.y, r.cy);
	rd.cz = scale(d.z, r.cz);
	M3 m;
	m.cx = v3(rd.cx.x * r.cx.x + rd.cy.x * r.cy.x + rd.cz.x * r.cz.x, rd.cx.y * r.cx.x + rd.cy.y * r.cy.x + rd.cz.y * r.cz.x,
			  rd.cx.z * r.cx.x + rd.cy.z * r.cy.x + rd.cz.z * r.cz.x);
	m.cy = v3(rd.cx.x * r.cx.y + rd.cy.x * r.cy.y + rd.cz.x * r.cz.y, rd.cx.y * r.cx.y + rd.cy.y * r.cy.y + rd.cz.y * r.cz.y,
			  rd.cx.z * r.cx.y + rd.cy.z * r.cy.y + rd.cz.z * r.cz.y);
	m.cz = v3(rd.cx.x * r.cx.z + rd.cy.x * r.cy.z + rd.cz.x * r.cz.z, rd.cx.y * r.cx.z + rd.cy.y * r.cy.z + rd.cz.y * r.cz.z,
			  rd.cx.z * r.cx.z + rd.cy.z * r.cy.z + rd.cz.z * r.cz.z);
	return m;
}

} // namespace m3g

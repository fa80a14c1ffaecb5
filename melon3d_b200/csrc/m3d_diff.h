// Differentiable substep: forward and reverse (adjoint) of the XPBD substep
// operations, templated on the scalar type.
//
// The forward functions restate the engine's element routines
// (m3d_solve.cuh; reference src/xpbd.cpp) with the same float operations in
// the same order, so with T = float they reproduce the engine bit for bit
// (the replay test checks that); with T = double the same code is the FP64
// host reference.  Each reverse function takes the adjoints of an
// operation's outputs and accumulates the adjoints of its inputs, recomputing
// the forward temporaries it needs.
//
// What is held fixed (the tape): the contact set, the solve order, which
// contacts had their manifold regenerated when (narrowphase or contact
// preparation), the feature ids of the points, which stiction anchors were
// kept or re-seated, and every branch the forward took (contact gates, caps,
// stiction, coherence and restitution tests, SAT axis and clipping choices).
// Derivatives flow through body states, inverse masses and inertias, friction
// and restitution coefficients, and through the manifold data as state: a
// manifold's normal, local anchors and separation offsets are functions of
// the poses it was generated at (m3d_diff_gen.h), stiction anchors start at
// the local anchors or carry over, and all of them persist across substeps
// and steps until the next generation (ContactBar carries their adjoint).
//
// Scope: spheres and boxes with isotropic inertia (cubes); no joints, no
// external forces; serial islands.  For an isotropic body the world inverse
// inertia R d R^T equals d I, so its derivative with respect to the rotation
// is zero and is not propagated.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define M3D_DIFF_HD __host__ __device__ __forceinline__
// a real call on the device: for the few large functions (the dual-number
// manifold generation) whose inlined copies would only cost registers and
// compile time
#define M3D_DIFF_HD_CALL __host__ __device__ __noinline__
#else
#define M3D_DIFF_HD inline
#define M3D_DIFF_HD_CALL inline
#endif

namespace m3d_diff
{

// ---- scalar functions with the engine's rounding for float -------------------

M3D_DIFF_HD float dsqrt(float x) { return sqrtf(x); }
M3D_DIFF_HD double dsqrt(double x) { return sqrt(x); }
// the engine evaluates these in double and rounds once
M3D_DIFF_HD float dsin(float x) { return (float)sin((double)x); }
M3D_DIFF_HD double dsin(double x) { return sin(x); }
M3D_DIFF_HD float dcos(float x) { return (float)cos((double)x); }
M3D_DIFF_HD double dcos(double x) { return cos(x); }
M3D_DIFF_HD float datan2(float y, float x) { return (float)atan2((double)y, (double)x); }
M3D_DIFF_HD double datan2(double y, double x) { return atan2(y, x); }
M3D_DIFF_HD float dabs(float x) { return fabsf(x); }
M3D_DIFF_HD double dabs(double x) { return fabs(x); }

template <typename T>
struct V
{
	T x, y, z;
};
template <typename T>
struct Q
{
	T x, y, z, w;
};
template <typename T>
struct M
{
	V<T> cx, cy, cz;
};

template <typename T>
M3D_DIFF_HD V<T> v3(T x, T y, T z)
{
	V<T> r;
	r.x = x;
	r.y = y;
	r.z = z;
	return r;
}
template <typename T>
M3D_DIFF_HD Q<T> q4(T x, T y, T z, T w)
{
	Q<T> r;
	r.x = x;
	r.y = y;
	r.z = z;
	r.w = w;
	return r;
}
template <typename T>
M3D_DIFF_HD V<T> vzero()
{
	return v3<T>(T(0), T(0), T(0));
}
template <typename T>
M3D_DIFF_HD Q<T> qzero()
{
	return q4<T>(T(0), T(0), T(0), T(0));
}
template <typename T>
M3D_DIFF_HD V<T> add(V<T> a, V<T> b)
{
	return v3<T>(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename T>
M3D_DIFF_HD V<T> sub(V<T> a, V<T> b)
{
	return v3<T>(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename T>
M3D_DIFF_HD V<T> neg(V<T> a)
{
	return v3<T>(-a.x, -a.y, -a.z);
}
template <typename T>
M3D_DIFF_HD V<T> scale(T s, V<T> v)
{
	return v3<T>(s * v.x, s * v.y, s * v.z);
}
template <typename T>
M3D_DIFF_HD V<T> madd(V<T> a, T s, V<T> b)
{
	return v3<T>(a.x + s * b.x, a.y + s * b.y, a.z + s * b.z);
}
template <typename T>
M3D_DIFF_HD T dot(V<T> a, V<T> b)
{
	return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T>
M3D_DIFF_HD V<T> cross(V<T> a, V<T> b)
{
	return v3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T>
M3D_DIFF_HD T len(V<T> v)
{
	return dsqrt(dot(v, v));
}
template <typename T>
M3D_DIFF_HD Q<T> qadd(Q<T> a, Q<T> b)
{
	return q4<T>(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
template <typename T>
M3D_DIFF_HD Q<T> qscale(T s, Q<T> a)
{
	return q4<T>(s * a.x, s * a.y, s * a.z, s * a.w);
}
template <typename T>
M3D_DIFF_HD T qdot(Q<T> a, Q<T> b)
{
	return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
template <typename T>
M3D_DIFF_HD Q<T> qmul(Q<T> a, Q<T> b)
{
	Q<T> q;
	q.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
	q.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
	q.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
	q.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
	return q;
}
template <typename T>
M3D_DIFF_HD Q<T> qconj(Q<T> q)
{
	return q4<T>(-q.x, -q.y, -q.z, q.w);
}
template <typename T>
M3D_DIFF_HD V<T> rotate(Q<T> q, V<T> v)
{
	V<T> u = v3<T>(q.x, q.y, q.z);
	V<T> t = scale(T(2), cross(u, v));
	return add(add(v, scale(q.w, t)), cross(u, t));
}
template <typename T>
M3D_DIFF_HD Q<T> renormFast(Q<T> q)
{
	T s = T(1.5) - T(0.5) * (q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
	return q4<T>(q.x * s, q.y * s, q.z * s, q.w * s);
}
template <typename T>
M3D_DIFF_HD V<T> mulv(const M<T>& m, V<T> v)
{
	return add(add(scale(v.x, m.cx), scale(v.y, m.cy)), scale(v.z, m.cz));
}
// I^-1_world = R diag(d) R^T, element order of the engine
template <typename T>
M3D_DIFF_HD M<T> invInertiaWorld(Q<T> q, V<T> d)
{
	T x = q.x, y = q.y, z = q.z, w = q.w;
	T x2 = x + x, y2 = y + y, z2 = z + z;
	T xx = x * x2, xy = x * y2, xz = x * z2;
	T yy = y * y2, yz = y * z2, zz = z * z2;
	T wx = w * x2, wy = w * y2, wz = w * z2;
	M<T> r;
	r.cx = v3<T>(T(1) - (yy + zz), xy + wz, xz - wy);
	r.cy = v3<T>(xy - wz, T(1) - (xx + zz), yz + wx);
	r.cz = v3<T>(xz + wy, yz - wx, T(1) - (xx + yy));
	M<T> rd;
	rd.cx = scale(d.x, r.cx);
	rd.cy = scale(d.y, r.cy);
	rd.cz = scale(d.z, r.cz);
	M<T> m;
	m.cx = v3<T>(rd.cx.x * r.cx.x + rd.cy.x * r.cy.x + rd.cz.x * r.cz.x, rd.cx.y * r.cx.x + rd.cy.y * r.cy.x + rd.cz.y * r.cz.x,
				 rd.cx.z * r.cx.x + rd.cy.z * r.cy.x + rd.cz.z * r.cz.x);
	m.cy = v3<T>(rd.cx.x * r.cx.y + rd.cy.x * r.cy.y + rd.cz.x * r.cz.y, rd.cx.y * r.cx.y + rd.cy.y * r.cy.y + rd.cz.y * r.cz.y,
				 rd.cx.z * r.cx.y + rd.cy.z * r.cy.y + rd.cz.z * r.cz.y);
	m.cz = v3<T>(rd.cx.x * r.cx.z + rd.cy.x * r.cy.z + rd.cz.x * r.cz.z, rd.cx.y * r.cx.z + rd.cy.y * r.cy.z + rd.cz.y * r.cz.z,
				 rd.cx.z * r.cx.z + rd.cy.z * r.cy.z + rd.cz.z * r.cz.z);
	return m;
}

// ---- reverse of the primitives ------------------------------------------------
// Each *_rev accumulates (+=) the adjoints of the inputs given the output's.

template <typename T>
M3D_DIFF_HD void cross_rev(V<T> a, V<T> b, V<T> o, V<T>& ab, V<T>& bb)
{
	// o . (da x b) = da . (b x o);  o . (a x db) = db . (o x a)
	ab = add(ab, cross(b, o));
	bb = add(bb, cross(o, a));
}
template <typename T>
M3D_DIFF_HD void qmul_rev(Q<T> a, Q<T> b, Q<T> o, Q<T>& ab, Q<T>& bb)
{
	// o = a (x) b is bilinear; the transposed rows of the product formula
	ab.x += o.x * b.w - o.y * b.z + o.z * b.y - o.w * b.x;
	ab.y += o.x * b.z + o.y * b.w - o.z * b.x - o.w * b.y;
	ab.z += -o.x * b.y + o.y * b.x + o.z * b.w - o.w * b.z;
	ab.w += o.x * b.x + o.y * b.y + o.z * b.z + o.w * b.w;
	bb.x += o.x * a.w + o.y * a.z - o.z * a.y - o.w * a.x;
	bb.y += -o.x * a.z + o.y * a.w + o.z * a.x - o.w * a.y;
	bb.z += o.x * a.y - o.y * a.x + o.z * a.w - o.w * a.z;
	bb.w += o.x * a.x + o.y * a.y + o.z * a.z + o.w * a.w;
}
template <typename T>
M3D_DIFF_HD void renormFast_rev(Q<T> q, Q<T> o, Q<T>& qb)
{
	// out = s q, s = 1.5 - 0.5 |q|^2:  d out = s dq - q (q . dq)
	T s = T(1.5) - T(0.5) * qdot(q, q);
	T k = qdot(o, q);
	qb.x += s * o.x - q.x * k;
	qb.y += s * o.y - q.y * k;
	qb.z += s * o.z - q.z * k;
	qb.w += s * o.w - q.w * k;
}
// rotate(q, v) with v constant: adjoint of q
template <typename T>
M3D_DIFF_HD void rotate_rev_q(Q<T> q, V<T> v, V<T> o, Q<T>& qb)
{
	V<T> u = v3<T>(q.x, q.y, q.z);
	V<T> t = scale(T(2), cross(u, v));
	// out = v + w t + u x t
	qb.w += dot(o, t);
	V<T> tb = scale(q.w, o);
	V<T> ub = vzero<T>();
	cross_rev(u, t, o, ub, tb);
	// t = 2 u x v
	V<T> vb = vzero<T>();
	cross_rev(u, v, scale(T(2), tb), ub, vb);
	qb.x += ub.x;
	qb.y += ub.y;
	qb.z += ub.z;
}
// adjoint of the rotated vector: rotate(q, v) is linear in v, M(q) v with
// M = I + 2w[u]x + 2[u]x^2; its transpose is the rotation by conj(q)
template <typename T>
M3D_DIFF_HD V<T> rotate_rev_v(Q<T> q, V<T> o)
{
	return rotate(qconj(q), o);
}
// y = m v: adjoints of m (outer product) and v
template <typename T>
M3D_DIFF_HD void mulv_rev(const M<T>& m, V<T> v, V<T> o, M<T>& mb, V<T>& vb)
{
	mb.cx = madd(mb.cx, v.x, o);
	mb.cy = madd(mb.cy, v.y, o);
	mb.cz = madd(mb.cz, v.z, o);
	vb.x += dot(m.cx, o);
	vb.y += dot(m.cy, o);
	vb.z += dot(m.cz, o);
}
// len(v): adjoint of v
template <typename T>
M3D_DIFF_HD void len_rev(V<T> v, T l, T ob, V<T>& vb)
{
	if (l > T(0))
	{
		vb = madd(vb, ob / l, v);
	}
}
// I^-1_world of an isotropic body: d (m) / d d = R R^T, taken as the identity
template <typename T>
M3D_DIFF_HD T iw_rev_isotropic(const M<T>& mb)
{
	return mb.cx.x + mb.cy.y + mb.cz.z;
}

// ---- per-body state ---------------------------------------------------------

template <typename T>
struct Body
{
	V<T> x;
	Q<T> q;
	V<T> v;
	V<T> w;
};
template <typename T>
M3D_DIFF_HD Body<T> bodyZero()
{
	Body<T> b;
	b.x = vzero<T>();
	b.q = qzero<T>();
	b.v = vzero<T>();
	b.w = vzero<T>();
	return b;
}
// constants of a body during the step (the isotropic inverse inertia `il` is
// one value; the engine stores it per axis, all three equal)
template <typename T>
struct BodyConst
{
	T invMass;
	T il;
	T gravityScale;
	T linearDamping;
	T angularDamping;
	int dynamic;
};
template <typename T>
struct BodyConstBar
{
	T invMass;
	T il;
};

// ---- integration (reference src/xpbd.cpp:587-705; isotropic: no gyroscopic
// term, no external force) ---------------------------------------------------

template <typename T>
M3D_DIFF_HD void integrate(const Body<T>& s0, const BodyConst<T>& c, T h, V<T> g, Body<T>& s1, M<T>& iw)
{
	V<T> v = madd(s0.v, h * c.gravityScale, g);
	V<T> w = s0.w;
	v = scale(T(1) / (T(1) + h * c.linearDamping), v);
	w = scale(T(1) / (T(1) + h * c.angularDamping), w);
	Q<T> q = s0.q;
	V<T> x = madd(s0.x, h, v);
	T wlen = len(w);
	if (wlen > T(1e-9))
	{
		T half = T(0.5) * h * wlen;
		T sinHalf, cosHalf;
		if (half < T(0.02))
		{
			T h2 = half * half;
			sinHalf = half * (T(1) - h2 * (T(1) / T(6)));
			cosHalf = T(1) - h2 * T(0.5);
		}
		else
		{
			sinHalf = dsin(half);
			cosHalf = dcos(half);
		}
		T s = sinHalf / wlen;
		Q<T> dq = q4<T>(w.x * s, w.y * s, w.z * s, cosHalf);
		q = renormFast(qmul(dq, q));
	}
	s1.x = x;
	s1.q = q;
	s1.v = v;
	s1.w = w;
	iw = invInertiaWorld(q, v3<T>(c.il, c.il, c.il));
}

// given the adjoints of s1 and iw, accumulate those of s0 and of il
template <typename T>
M3D_DIFF_HD void integrate_rev(const Body<T>& s0, const BodyConst<T>& c, T h, V<T> g, const Body<T>& s1b,
							   const M<T>& iwb, Body<T>& s0b, BodyConstBar<T>& cb)
{
	const T cl = T(1) / (T(1) + h * c.linearDamping);
	const T ca = T(1) / (T(1) + h * c.angularDamping);
	V<T> w = scale(ca, s0.w);
	// x1 = x0 + h v1, v1 = cl (v0 + h gs g)
	V<T> vb = madd(s1b.v, h, s1b.x);
	s0b.x = add(s0b.x, s1b.x);
	s0b.v = madd(s0b.v, cl, vb);
	V<T> wb = s1b.w;
	T wlen = len(w);
	if (wlen > T(1e-9))
	{
		T half = T(0.5) * h * wlen;
		T sinHalf, cosHalf, dsin_dh, dcos_dh;
		if (half < T(0.02))
		{
			T h2 = half * half;
			sinHalf = half * (T(1) - h2 * (T(1) / T(6)));
			cosHalf = T(1) - h2 * T(0.5);
			dsin_dh = T(1) - half * half * T(0.5);
			dcos_dh = -half;
		}
		else
		{
			sinHalf = dsin(half);
			cosHalf = dcos(half);
			dsin_dh = cosHalf;
			dcos_dh = -sinHalf;
		}
		T s = sinHalf / wlen;
		Q<T> dq = q4<T>(w.x * s, w.y * s, w.z * s, cosHalf);
		Q<T> p = qmul(dq, s0.q);
		Q<T> pb = qzero<T>();
		renormFast_rev(p, s1b.q, pb);
		Q<T> dqb = qzero<T>();
		qmul_rev(dq, s0.q, pb, dqb, s0b.q);
		// dq = (w s, cosHalf)
		wb = madd(wb, s, v3<T>(dqb.x, dqb.y, dqb.z));
		T sb = w.x * dqb.x + w.y * dqb.y + w.z * dqb.z;
		T halfb = dqb.w * dcos_dh + (sb / wlen) * dsin_dh;
		T wlenb = -sb * sinHalf / (wlen * wlen) + T(0.5) * h * halfb;
		len_rev(w, wlen, wlenb, wb);
	}
	else
	{
		// no spin: the engine leaves the rotation as it is.  The rotation is
		// still a smooth function of the spin through zero (any spin takes
		// the small-angle branch, q1 = q0 + h/2 (w, 0) q0 to first order), so
		// the spin's adjoint is that branch's limit.
		s0b.q = qadd(s0b.q, s1b.q);
		Q<T> dqb = qzero<T>(), unused = qzero<T>();
		qmul_rev(q4<T>(T(0), T(0), T(0), T(1)), s0.q, s1b.q, dqb, unused);
		wb = madd(wb, T(0.5) * h, v3<T>(dqb.x, dqb.y, dqb.z));
	}
	s0b.w = madd(s0b.w, ca, wb);
	cb.il += iw_rev_isotropic(iwb);
}

// ---- contacts -------------------------------------------------------------

enum ShapeKind
{
	kShapeSphere = 0,
	kShapeBox = 2
};

// the frozen manifold of one contact in one substep (as left by contact
// preparation), with its materials
template <typename T>
struct Contact
{
	int a, b;          // body indices (island-local or global, as the caller uses them)
	int pointCount;
	int curved;        // not box-box: the velocity pass recomputes arms
	int shapeA, shapeB;
	T radiusA, radiusB;
	V<T> n;
	T mu, e, rolling;
	V<T> la[4], lb[4]; // local anchors
	T off[4];          // separation offsets
	V<T> fa[4], fb[4]; // stiction anchors
	V<T> slip[4];      // slip directions of the last velocity pass
};

// adjoint of a contact's manifold data: normal, local anchors, separation
// offsets, stiction anchors (the fields every substep reads)
template <typename T>
struct ContactBar
{
	V<T> n;
	V<T> la[4], lb[4], fa[4], fb[4];
	T off[4];
};
template <typename T>
M3D_DIFF_HD void contactBarZero(ContactBar<T>& b)
{
	b.n = vzero<T>();
	for (int s = 0; s < 4; ++s)
	{
		b.la[s] = b.lb[s] = b.fa[s] = b.fb[s] = vzero<T>();
		b.off[s] = T(0);
	}
}

// contact quantities frozen at preparation (reference src/xpbd.cpp:733-863)
template <typename T>
struct Prepared
{
	V<T> rA[4], rB[4], jA[4], jB[4];
	T wN[4];
};
template <typename T>
M3D_DIFF_HD void preparedZero(Prepared<T>& p)
{
	for (int s = 0; s < 4; ++s)
	{
		p.rA[s] = p.rB[s] = p.jA[s] = p.jB[s] = vzero<T>();
		p.wN[s] = T(0);
	}
}

// contact arm: geometric for a sphere, the rotated anchor for a box
template <typename T>
M3D_DIFF_HD V<T> arm(int shape, T radius, Q<T> q, V<T> l, V<T> n, T sign)
{
	return shape == kShapeSphere ? scale(sign * radius, n) : rotate(q, l);
}
template <typename T>
M3D_DIFF_HD void arm_rev(int shape, T radius, Q<T> q, V<T> l, T sign, V<T> rb, Q<T>& qb, V<T>& lb, V<T>& nb)
{
	if (shape != kShapeSphere)
	{
		rotate_rev_q(q, l, rb, qb);
		lb = add(lb, rotate_rev_v(q, rb));
	}
	else
	{
		nb = madd(nb, sign * radius, rb);
	}
}

template <typename T>
M3D_DIFF_HD void prepare(const Contact<T>& c, Q<T> qA, Q<T> qB, T imA, T imB, const M<T>& iwA, const M<T>& iwB,
						 Prepared<T>& p)
{
	for (int s = 0; s < c.pointCount; ++s)
	{
		V<T> rA = arm(c.shapeA, c.radiusA, qA, c.la[s], c.n, T(1));
		V<T> rB = arm(c.shapeB, c.radiusB, qB, c.lb[s], c.n, T(-1));
		V<T> crossA = cross(rA, c.n);
		V<T> crossB = cross(rB, c.n);
		V<T> jA = mulv(iwA, crossA);
		V<T> jB = mulv(iwB, crossB);
		p.rA[s] = rA;
		p.rB[s] = rB;
		p.jA[s] = jA;
		p.jB[s] = jB;
		p.wN[s] = imA + imB + dot(crossA, jA) + dot(crossB, jB);
	}
}

template <typename T>
M3D_DIFF_HD void prepare_rev(const Contact<T>& c, Q<T> qA, Q<T> qB, const M<T>& iwA, const M<T>& iwB,
							 const Prepared<T>& p, const Prepared<T>& pb, Q<T>& qAb, Q<T>& qBb, T& imAb, T& imBb,
							 M<T>& iwAb, M<T>& iwBb, ContactBar<T>& cb)
{
	for (int s = 0; s < c.pointCount; ++s)
	{
		V<T> crossA = cross(p.rA[s], c.n);
		V<T> crossB = cross(p.rB[s], c.n);
		T wb = pb.wN[s];
		imAb += wb;
		imBb += wb;
		V<T> cAb = scale(wb, p.jA[s]);
		V<T> cBb = scale(wb, p.jB[s]);
		V<T> jAb = madd(pb.jA[s], wb, crossA);
		V<T> jBb = madd(pb.jB[s], wb, crossB);
		mulv_rev(iwA, crossA, jAb, iwAb, cAb);
		mulv_rev(iwB, crossB, jBb, iwBb, cBb);
		V<T> rAb = pb.rA[s], rBb = pb.rB[s];
		cross_rev(p.rA[s], c.n, cAb, rAb, cb.n);
		cross_rev(p.rB[s], c.n, cBb, rBb, cb.n);
		arm_rev(c.shapeA, c.radiusA, qA, c.la[s], T(1), rAb, qAb, cb.la[s], cb.n);
		arm_rev(c.shapeB, c.radiusB, qB, c.lb[s], T(-1), rBb, qBb, cb.lb[s], cb.n);
	}
}

// ApplyAxisCorrection (reference src/xpbd.cpp:45-58)
template <typename T>
M3D_DIFF_HD void axisCorrection(V<T>& p, Q<T>& q, T im, T dl, V<T> n, V<T> j)
{
	if (im == T(0))
	{
		return;
	}
	p = madd(p, dl * im, n);
	V<T> dw = scale(dl, j);
	Q<T> dq = qmul(q4<T>(dw.x, dw.y, dw.z, T(0)), q);
	q = renormFast(q4<T>(q.x + T(0.5) * dq.x, q.y + T(0.5) * dq.y, q.z + T(0.5) * dq.z, q.w + T(0.5) * dq.w));
}
// inputs p, q (before); adjoints pb, qb of the outputs in, of the inputs out
template <typename T>
M3D_DIFF_HD void axisCorrection_rev(Q<T> q, T im, T dl, V<T> n, V<T> j, V<T>& pb, Q<T>& qb, T& dlb, T& imb, V<T>& jb,
									V<T>& nb)
{
	if (im == T(0))
	{
		return;
	}
	nb = madd(nb, dl * im, pb);
	T s1b = dot(pb, n);
	dlb += s1b * im;
	imb += s1b * dl;
	V<T> dw = scale(dl, j);
	Q<T> wq = q4<T>(dw.x, dw.y, dw.z, T(0));
	Q<T> dq = qmul(wq, q);
	Q<T> P = q4<T>(q.x + T(0.5) * dq.x, q.y + T(0.5) * dq.y, q.z + T(0.5) * dq.z, q.w + T(0.5) * dq.w);
	Q<T> Pb = qzero<T>();
	renormFast_rev(P, qb, Pb);
	Q<T> wqb = qzero<T>();
	Q<T> qin = Pb;
	qmul_rev(wq, q, qscale(T(0.5), Pb), wqb, qin);
	qb = qin;
	V<T> dwb = v3<T>(wqb.x, wqb.y, wqb.z);
	dlb += dot(dwb, j);
	jb = madd(jb, dl, dwb);
}

// SolveContactNormals, serial form (reference src/xpbd.cpp:122-163): the
// points in order, each against the poses the previous one left
template <typename T>
M3D_DIFF_HD void normals(const Contact<T>& c, const Prepared<T>& p, T imA, T imB, T maxCorrection, V<T>& pA, Q<T>& qA,
						 V<T>& pB, Q<T>& qB, T* lambdaN)
{
	for (int s = 0; s < c.pointCount; ++s)
	{
		T wN = p.wN[s];
		if (wN <= T(0))
		{
			continue;
		}
		V<T> rA = rotate(qA, c.la[s]);
		V<T> rB = rotate(qB, c.lb[s]);
		T sep = c.off[s] + dot(sub(add(pB, rB), add(pA, rA)), c.n);
		if (sep >= T(0))
		{
			continue;
		}
		if (sep < -maxCorrection)
		{
			sep = -maxCorrection;
		}
		T dl = -sep / wN;
		lambdaN[s] += dl;
		axisCorrection(pB, qB, imB, dl, c.n, p.jB[s]);
		axisCorrection(pA, qA, imA, -dl, c.n, p.jA[s]);
	}
}

// adjoints of the poses after the op in (pAb ...), of the poses before out;
// lambdaNb: adjoint of each point's accumulated lambda (passes through)
template <typename T>
M3D_DIFF_HD void normals_rev(const Contact<T>& c, const Prepared<T>& p, T imA, T imB, T maxCorrection, V<T> pA0, Q<T> qA0,
							 V<T> pB0, Q<T> qB0, V<T>& pAb, Q<T>& qAb, V<T>& pBb, Q<T>& qBb, const T* lambdaNb,
							 Prepared<T>& pb, T& imAb, T& imBb, ContactBar<T>& cb)
{
	// poses before each point
	V<T> sA[4], sB[4];
	Q<T> tA[4], tB[4];
	V<T> pA = pA0, pB = pB0;
	Q<T> qA = qA0, qB = qB0;
	for (int s = 0; s < c.pointCount; ++s)
	{
		sA[s] = pA;
		tA[s] = qA;
		sB[s] = pB;
		tB[s] = qB;
		T wN = p.wN[s];
		if (wN <= T(0))
		{
			continue;
		}
		V<T> rA = rotate(qA, c.la[s]);
		V<T> rB = rotate(qB, c.lb[s]);
		T sep = c.off[s] + dot(sub(add(pB, rB), add(pA, rA)), c.n);
		if (sep >= T(0))
		{
			continue;
		}
		if (sep < -maxCorrection)
		{
			sep = -maxCorrection;
		}
		T dl = -sep / wN;
		axisCorrection(pB, qB, imB, dl, c.n, p.jB[s]);
		axisCorrection(pA, qA, imA, -dl, c.n, p.jA[s]);
	}
	for (int s = c.pointCount - 1; s >= 0; --s)
	{
		T wN = p.wN[s];
		if (wN <= T(0))
		{
			continue;
		}
		pA = sA[s];
		qA = tA[s];
		pB = sB[s];
		qB = tB[s];
		V<T> rA = rotate(qA, c.la[s]);
		V<T> rB = rotate(qB, c.lb[s]);
		T sep = c.off[s] + dot(sub(add(pB, rB), add(pA, rA)), c.n);
		if (sep >= T(0))
		{
			continue;
		}
		bool capped = sep < -maxCorrection;
		if (capped)
		{
			sep = -maxCorrection;
		}
		T dl = -sep / wN;
		// B was corrected first, A second: reverse A, then B
		T dlAb = T(0), dlBb = T(0);
		axisCorrection_rev(qA, imA, -dl, c.n, p.jA[s], pAb, qAb, dlAb, imAb, pb.jA[s], cb.n);
		axisCorrection_rev(qB, imB, dl, c.n, p.jB[s], pBb, qBb, dlBb, imBb, pb.jB[s], cb.n);
		T dlb = dlBb - dlAb + lambdaNb[s];
		T sepb = T(0);
		if (capped)
		{
			pb.wN[s] += -dlb * maxCorrection / (wN * wN);
		}
		else
		{
			sepb = -dlb / wN;
			pb.wN[s] += dlb * sep / (wN * wN);
		}
		V<T> gb = scale(sepb, c.n);
		pBb = add(pBb, gb);
		pAb = sub(pAb, gb);
		rotate_rev_q(qB, c.lb[s], gb, qBb);
		rotate_rev_q(qA, c.la[s], neg(gb), qAb);
		cb.off[s] += sepb;
		cb.n = madd(cb.n, sepb, sub(add(pB, rB), add(pA, rA)));
		cb.lb[s] = add(cb.lb[s], rotate_rev_v(qB, gb));
		cb.la[s] = sub(cb.la[s], rotate_rev_v(qA, gb));
	}
}

// ReconstructBodyVelocity (reference src/xpbd.cpp:865-892)
template <typename T>
M3D_DIFF_HD void reconstruct(V<T> x, Q<T> q, V<T> x0, Q<T> q0, T invH, V<T>& v, V<T>& w)
{
	v = scale(invH, sub(x, x0));
	Q<T> dq = qmul(q, qconj(q0));
	T sign = dq.w >= T(0) ? T(1) : T(-1);
	T v2 = dq.x * dq.x + dq.y * dq.y + dq.z * dq.z;
	if (v2 > T(4e-4))
	{
		T vl = dsqrt(v2);
		T angle = T(2) * datan2(vl, dabs(dq.w));
		w = scale(sign * invH * angle / vl, v3<T>(dq.x, dq.y, dq.z));
	}
	else
	{
		T corr = T(1) + v2 * (T(1) / T(6));
		w = scale(T(2) * invH * sign * corr, v3<T>(dq.x, dq.y, dq.z));
	}
}

template <typename T>
M3D_DIFF_HD void reconstruct_rev(V<T> x, Q<T> q, V<T> x0, Q<T> q0, T invH, V<T> vb, V<T> wb, V<T>& xb, Q<T>& qb,
								 V<T>& x0b, Q<T>& q0b)
{
	xb = madd(xb, invH, vb);
	x0b = madd(x0b, -invH, vb);
	Q<T> c0 = qconj(q0);
	Q<T> dq = qmul(q, c0);
	V<T> dv = v3<T>(dq.x, dq.y, dq.z);
	T sign = dq.w >= T(0) ? T(1) : T(-1);
	T v2 = dot(dv, dv);
	V<T> dvb = vzero<T>();
	T dwb = T(0);
	if (v2 > T(4e-4))
	{
		T vl = dsqrt(v2);
		T aw = dabs(dq.w);
		T angle = T(2) * datan2(vl, aw);
		T k = sign * invH * angle / vl;
		dvb = scale(k, wb);
		T kb = dot(wb, dv);
		T angleb = kb * sign * invH / vl;
		T vlb = -kb * sign * invH * angle / (vl * vl);
		T den = vl * vl + aw * aw;
		vlb += angleb * T(2) * aw / den;
		T awb = -angleb * T(2) * vl / den;
		dwb += awb * sign;
		T v2b = vlb / (T(2) * vl);
		dvb = madd(dvb, T(2) * v2b, dv);
	}
	else
	{
		T corr = T(1) + v2 * (T(1) / T(6));
		T k = T(2) * invH * sign * corr;
		dvb = scale(k, wb);
		T kb = dot(wb, dv);
		T corrb = kb * T(2) * invH * sign;
		T v2b = corrb / T(6);
		dvb = madd(dvb, T(2) * v2b, dv);
	}
	Q<T> dqb = q4<T>(dvb.x, dvb.y, dvb.z, dwb);
	Q<T> c0b = qzero<T>();
	qmul_rev(q, c0, dqb, qb, c0b);
	q0b.x -= c0b.x;
	q0b.y -= c0b.y;
	q0b.z -= c0b.z;
	q0b.w += c0b.w;
}

// generalised inverse mass along an axis: im + (r x a) . I^-1 (r x a)
template <typename T>
M3D_DIFF_HD T genInvMass(T im, const M<T>& iw, V<T> r, V<T> a)
{
	V<T> rn = cross(r, a);
	return im + dot(rn, mulv(iw, rn));
}
template <typename T>
M3D_DIFF_HD void genInvMass_rev(const M<T>& iw, V<T> r, V<T> a, T ob, T& imb, M<T>& iwb, V<T>& rb, V<T>& ab)
{
	V<T> rn = cross(r, a);
	V<T> y = mulv(iw, rn);
	imb += ob;
	V<T> rnb = scale(ob, y);
	mulv_rev(iw, rn, scale(ob, rn), iwb, rnb);
	cross_rev(r, a, rnb, rb, ab);
}

// ApplyPositionCorrection (reference src/xpbd.cpp:28-41)
template <typename T>
M3D_DIFF_HD void positionCorrection(V<T>& p, Q<T>& q, T im, const M<T>& iw, V<T> imp, V<T> r)
{
	if (im == T(0))
	{
		return;
	}
	p = madd(p, im, imp);
	V<T> dw = mulv(iw, cross(r, imp));
	Q<T> dq = qmul(q4<T>(dw.x, dw.y, dw.z, T(0)), q);
	q = renormFast(q4<T>(q.x + T(0.5) * dq.x, q.y + T(0.5) * dq.y, q.z + T(0.5) * dq.z, q.w + T(0.5) * dq.w));
}
template <typename T>
M3D_DIFF_HD void positionCorrection_rev(Q<T> q, T im, const M<T>& iw, V<T> imp, V<T> r, V<T>& pb, Q<T>& qb, T& imb,
										M<T>& iwb, V<T>& impb, V<T>& rb)
{
	if (im == T(0))
	{
		return;
	}
	impb = madd(impb, im, pb);
	imb += dot(pb, imp);
	V<T> c = cross(r, imp);
	V<T> dw = mulv(iw, c);
	Q<T> wq = q4<T>(dw.x, dw.y, dw.z, T(0));
	Q<T> dq = qmul(wq, q);
	Q<T> P = q4<T>(q.x + T(0.5) * dq.x, q.y + T(0.5) * dq.y, q.z + T(0.5) * dq.z, q.w + T(0.5) * dq.w);
	Q<T> Pb = qzero<T>();
	renormFast_rev(P, qb, Pb);
	Q<T> wqb = qzero<T>();
	Q<T> qin = Pb;
	qmul_rev(wq, q, qscale(T(0.5), Pb), wqb, qin);
	qb = qin;
	V<T> cb = vzero<T>();
	mulv_rev(iw, c, v3<T>(wqb.x, wqb.y, wqb.z), iwb, cb);
	cross_rev(r, imp, cb, rb, impb);
}

// ApplyContactFriction, positional stiction toward the anchors, box-box
// only (reference src/xpbd.cpp:172-269).  Returns false when the speed gate
// re-anchored the contact instead (nothing moves).
template <typename T>
M3D_DIFF_HD bool frictionGate(const Contact<T>& c, const Prepared<T>& p, V<T> va, V<T> wa, V<T> vb, V<T> wb)
{
	if (c.shapeA != kShapeBox || c.shapeB != kShapeBox || c.pointCount == 0)
	{
		return false;
	}
	V<T> vrel = sub(add(vb, cross(wb, p.rB[0])), add(va, cross(wa, p.rA[0])));
	V<T> vt = sub(vrel, scale(dot(vrel, c.n), c.n));
	return !(dot(vt, vt) > T(0.1) * T(0.1));
}

// resetMask (optional) receives the points whose anchors the engine re-seats
// at the local anchors after this pass (needed > 2 allowed)
template <typename T>
M3D_DIFF_HD void friction(const Contact<T>& c, T imA, T imB, const M<T>& iwA, const M<T>& iwB, const T* lambdaN,
						  V<T>& pA, Q<T>& qA, V<T>& pB, Q<T>& qB, T* lambdaT, int* resetMask = nullptr)
{
	for (int s = 0; s < c.pointCount; ++s)
	{
		T lN = lambdaN[s];
		if (lN <= T(0))
		{
			continue;
		}
		V<T> rA = rotate(qA, c.fa[s]);
		V<T> rB = rotate(qB, c.fb[s]);
		V<T> gap = sub(add(pB, rB), add(pA, rA));
		V<T> dpt = sub(gap, scale(dot(gap, c.n), c.n));
		T lt = len(dpt);
		if (lt <= T(1e-9))
		{
			continue;
		}
		V<T> t = scale(T(1) / lt, dpt);
		T wt = genInvMass(imA, iwA, rA, t) + genInvMass(imB, iwB, rB, t);
		if (wt <= T(0))
		{
			continue;
		}
		T needed = T(0.5) * (lt / wt);
		T allowed = c.mu * lN - lambdaT[s];
		if (allowed <= T(0))
		{
			continue;
		}
		T dL = needed < allowed ? needed : allowed;
		lambdaT[s] += dL;
		V<T> pt = scale(dL, t);
		positionCorrection(pB, qB, imB, iwB, neg(pt), rB);
		positionCorrection(pA, qA, imA, iwA, pt, rA);
		if (resetMask != nullptr && needed > T(2) * allowed)
		{
			*resetMask |= 1 << s;
		}
	}
}

template <typename T>
M3D_DIFF_HD void friction_rev(const Contact<T>& c, T imA, T imB, const M<T>& iwA, const M<T>& iwB, const T* lambdaN,
							  V<T> pA0, Q<T> qA0, V<T> pB0, Q<T> qB0, const T* lambdaT0, V<T>& pAb, Q<T>& qAb,
							  V<T>& pBb, Q<T>& qBb, T* lambdaNb, T* lambdaTb, T& muB, T& imAb, T& imBb, M<T>& iwAb,
							  M<T>& iwBb, ContactBar<T>& cb)
{
	V<T> sA[4], sB[4];
	Q<T> tA[4], tB[4];
	T lT[4];
	V<T> pA = pA0, pB = pB0;
	Q<T> qA = qA0, qB = qB0;
	for (int s = 0; s < 4; ++s)
	{
		lT[s] = lambdaT0[s];
	}
	for (int s = 0; s < c.pointCount; ++s)
	{
		sA[s] = pA;
		tA[s] = qA;
		sB[s] = pB;
		tB[s] = qB;
		T lN = lambdaN[s];
		if (lN <= T(0))
		{
			continue;
		}
		V<T> rA = rotate(qA, c.fa[s]);
		V<T> rB = rotate(qB, c.fb[s]);
		V<T> gap = sub(add(pB, rB), add(pA, rA));
		V<T> dpt = sub(gap, scale(dot(gap, c.n), c.n));
		T lt = len(dpt);
		if (lt <= T(1e-9))
		{
			continue;
		}
		V<T> t = scale(T(1) / lt, dpt);
		T wt = genInvMass(imA, iwA, rA, t) + genInvMass(imB, iwB, rB, t);
		if (wt <= T(0))
		{
			continue;
		}
		T needed = T(0.5) * (lt / wt);
		T allowed = c.mu * lN - lT[s];
		if (allowed <= T(0))
		{
			continue;
		}
		T dL = needed < allowed ? needed : allowed;
		lT[s] += dL;
		V<T> pt = scale(dL, t);
		positionCorrection(pB, qB, imB, iwB, neg(pt), rB);
		positionCorrection(pA, qA, imA, iwA, pt, rA);
	}
	for (int s = c.pointCount - 1; s >= 0; --s)
	{
		T lN = lambdaN[s];
		if (lN <= T(0))
		{
			continue;
		}
		pA = sA[s];
		qA = tA[s];
		pB = sB[s];
		qB = tB[s];
		T lT0 = lambdaT0[s];
		V<T> rA = rotate(qA, c.fa[s]);
		V<T> rB = rotate(qB, c.fb[s]);
		V<T> gap = sub(add(pB, rB), add(pA, rA));
		T gn = dot(gap, c.n);
		V<T> dpt = sub(gap, scale(gn, c.n));
		T lt = len(dpt);
		if (lt <= T(1e-9))
		{
			continue;
		}
		T inv = T(1) / lt;
		V<T> t = scale(inv, dpt);
		T wt = genInvMass(imA, iwA, rA, t) + genInvMass(imB, iwB, rB, t);
		if (wt <= T(0))
		{
			continue;
		}
		T needed = T(0.5) * (lt / wt);
		T allowed = c.mu * lN - lT0;
		if (allowed <= T(0))
		{
			continue;
		}
		bool takeNeeded = needed < allowed;
		T dL = takeNeeded ? needed : allowed;
		V<T> pt = scale(dL, t);
		// reverse: A's correction (last), then B's
		V<T> ptb = vzero<T>(), rAb = vzero<T>(), rBb = vzero<T>();
		positionCorrection_rev(qA, imA, iwA, pt, rA, pAb, qAb, imAb, iwAb, ptb, rAb);
		V<T> nptb = vzero<T>();
		positionCorrection_rev(qB, imB, iwB, neg(pt), rB, pBb, qBb, imBb, iwBb, nptb, rBb);
		ptb = sub(ptb, nptb);
		T dLb = dot(ptb, t) + lambdaTb[s];
		V<T> tb = scale(dL, ptb);
		T neededb = T(0), allowedb = T(0);
		if (takeNeeded)
			neededb = dLb;
		else
			allowedb = dLb;
		muB += allowedb * lN;
		lambdaNb[s] += allowedb * c.mu;
		lambdaTb[s] -= allowedb;
		T ltb = neededb * T(0.5) / wt;
		T wtb = -neededb * T(0.5) * lt / (wt * wt);
		genInvMass_rev(iwA, rA, t, wtb, imAb, iwAb, rAb, tb);
		genInvMass_rev(iwB, rB, t, wtb, imBb, iwBb, rBb, tb);
		// t = inv dpt, inv = 1/lt
		V<T> dptb = scale(inv, tb);
		ltb += -dot(tb, dpt) * inv * inv;
		len_rev(dpt, lt, ltb, dptb);
		// dpt = gap - (gap.n) n
		T ndp = dot(dptb, c.n);
		V<T> gapb = sub(dptb, scale(ndp, c.n));
		cb.n = sub(cb.n, add(scale(gn, dptb), scale(ndp, gap)));
		pBb = add(pBb, gapb);
		pAb = sub(pAb, gapb);
		rBb = add(rBb, gapb);
		rAb = sub(rAb, gapb);
		rotate_rev_q(qA, c.fa[s], rAb, qAb);
		rotate_rev_q(qB, c.fb[s], rBb, qBb);
		cb.fa[s] = add(cb.fa[s], rotate_rev_v(qA, rAb));
		cb.fb[s] = add(cb.fb[s], rotate_rev_v(qB, rBb));
	}
}

// SolveContactVelocity (reference src/xpbd.cpp:275-407): dynamic friction
// with the coherence test, restitution against the pre-substep normal
// velocity, the normal-velocity fix, rolling resistance.  Velocities in/out;
// qA, qB are the current rotations (curved arms); pv*, pw* the velocities at
// the start of the substep.
template <typename T>
struct VelocityIn
{
	T imA, imB;
	M<T> iwA, iwB;
	Q<T> qA, qB;
	V<T> pva, pwa, pvb, pwb;
	T h, gravityLen;
};

template <typename T>
M3D_DIFF_HD void velocity(const Contact<T>& c, const Prepared<T>& p, const VelocityIn<T>& in, const T* lambdaN, V<T>& va,
						  V<T>& wa, V<T>& vb, V<T>& wb)
{
	const T invH = in.h > T(0) ? T(1) / in.h : T(0);
	T lambdaNTotal = T(0);
	for (int s = 0; s < c.pointCount; ++s)
	{
		T lN = lambdaN[s];
		if (lN <= T(0))
		{
			continue;
		}
		V<T> rAf, rBf;
		if (c.curved)
		{
			rAf = arm(c.shapeA, c.radiusA, in.qA, c.la[s], c.n, T(1));
			rBf = arm(c.shapeB, c.radiusB, in.qB, c.lb[s], c.n, T(-1));
		}
		else
		{
			rAf = p.rA[s];
			rBf = p.rB[s];
		}
		V<T> vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		T vn = dot(vrel, c.n);
		V<T> vt = sub(vrel, scale(vn, c.n));
		T vtLen = len(vt);
		if (vtLen > T(1e-9))
		{
			V<T> t = scale(T(1) / vtLen, vt);
			T wt = genInvMass(in.imA, in.iwA, rAf, t) + genInvMass(in.imB, in.iwB, rBf, t);
			if (wt > T(0))
			{
				bool coherent = dot(t, c.slip[s]) > T(0.7);
				T pStop = vtLen / wt;
				T pMax = c.mu * lN * invH;
				T P = !coherent && vtLen < T(0.08) ? pStop : (pStop < pMax ? pStop : pMax);
				V<T> imp = scale(-P, t);
				if (in.imB != T(0))
				{
					vb = madd(vb, in.imB, imp);
					wb = add(wb, mulv(in.iwB, cross(rBf, imp)));
				}
				if (in.imA != T(0))
				{
					V<T> pn = neg(imp);
					va = madd(va, in.imA, pn);
					wa = add(wa, mulv(in.iwA, cross(rAf, pn)));
				}
			}
		}
		V<T> vrelPrev = sub(add(in.pvb, cross(in.pwb, rBf)), add(in.pva, cross(in.pwa, rAf)));
		T vnPrev = dot(vrelPrev, c.n);
		T e = dabs(vnPrev) > T(2) * in.gravityLen * in.h ? c.e : T(0);
		vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		vn = dot(vrel, c.n);
		T target = -e * vnPrev;
		target = target > T(0) ? target : T(0);
		T wN = p.wN[s];
		if (wN > T(0))
		{
			T j = (target - vn) / wN;
			if (in.imB != T(0))
			{
				vb = madd(vb, j * in.imB, c.n);
				wb = madd(wb, j, p.jB[s]);
			}
			if (in.imA != T(0))
			{
				T mj = -j;
				va = madd(va, mj * in.imA, c.n);
				wa = madd(wa, mj, p.jA[s]);
			}
		}
		lambdaNTotal += lN > T(0) ? lN : T(0);
	}
	if (c.rolling > T(0) && lambdaNTotal > T(0))
	{
		V<T> wrel = sub(wb, wa);
		V<T> wroll = sub(wrel, scale(dot(wrel, c.n), c.n));
		T wl = len(wroll);
		if (wl > T(1e-6))
		{
			V<T> axis = scale(T(1) / wl, wroll);
			T kk = dot(axis, mulv(in.iwA, axis)) + dot(axis, mulv(in.iwB, axis));
			if (kk > T(1e-12))
			{
				T maxDw = c.rolling * lambdaNTotal * invH * kk;
				T dw = maxDw < wl ? maxDw : wl;
				V<T> angImp = scale(dw / kk, axis);
				wb = sub(wb, mulv(in.iwB, angImp));
				wa = add(wa, mulv(in.iwA, angImp));
			}
		}
	}
}

// adjoints accumulated by the velocity pass of one contact
template <typename T>
struct VelocityBar
{
	T imA, imB, mu, e;
	M<T> iwA, iwB;
	Q<T> qA, qB;
	V<T> pva, pwa, pvb, pwb;
};

template <typename T>
M3D_DIFF_HD void velocity_rev(const Contact<T>& c, const Prepared<T>& p, const VelocityIn<T>& in, const T* lambdaN,
							  V<T> va0, V<T> wa0, V<T> vb0, V<T> wb0, V<T>& vab, V<T>& wab, V<T>& vbb, V<T>& wbb,
							  Prepared<T>& pb, T* lambdaNb, VelocityBar<T>& b, ContactBar<T>& cb)
{
	const T invH = in.h > T(0) ? T(1) / in.h : T(0);
	// forward, keeping the velocities before each point
	V<T> sva[4], swa[4], svb[4], swb[4];
	V<T> va = va0, wa = wa0, vb = vb0, wb = wb0;
	T lambdaNTotal = T(0);
	for (int s = 0; s < c.pointCount; ++s)
	{
		sva[s] = va;
		swa[s] = wa;
		svb[s] = vb;
		swb[s] = wb;
		T lN = lambdaN[s];
		if (lN <= T(0))
		{
			continue;
		}
		V<T> rAf, rBf;
		if (c.curved)
		{
			rAf = arm(c.shapeA, c.radiusA, in.qA, c.la[s], c.n, T(1));
			rBf = arm(c.shapeB, c.radiusB, in.qB, c.lb[s], c.n, T(-1));
		}
		else
		{
			rAf = p.rA[s];
			rBf = p.rB[s];
		}
		V<T> vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		T vn = dot(vrel, c.n);
		V<T> vt = sub(vrel, scale(vn, c.n));
		T vtLen = len(vt);
		if (vtLen > T(1e-9))
		{
			V<T> t = scale(T(1) / vtLen, vt);
			T wt = genInvMass(in.imA, in.iwA, rAf, t) + genInvMass(in.imB, in.iwB, rBf, t);
			if (wt > T(0))
			{
				bool coherent = dot(t, c.slip[s]) > T(0.7);
				T pStop = vtLen / wt;
				T pMax = c.mu * lN * invH;
				T P = !coherent && vtLen < T(0.08) ? pStop : (pStop < pMax ? pStop : pMax);
				V<T> imp = scale(-P, t);
				if (in.imB != T(0))
				{
					vb = madd(vb, in.imB, imp);
					wb = add(wb, mulv(in.iwB, cross(rBf, imp)));
				}
				if (in.imA != T(0))
				{
					V<T> pn = neg(imp);
					va = madd(va, in.imA, pn);
					wa = add(wa, mulv(in.iwA, cross(rAf, pn)));
				}
			}
		}
		V<T> vrelPrev = sub(add(in.pvb, cross(in.pwb, rBf)), add(in.pva, cross(in.pwa, rAf)));
		T vnPrev = dot(vrelPrev, c.n);
		T e = dabs(vnPrev) > T(2) * in.gravityLen * in.h ? c.e : T(0);
		vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		vn = dot(vrel, c.n);
		T target = -e * vnPrev;
		target = target > T(0) ? target : T(0);
		T wN = p.wN[s];
		if (wN > T(0))
		{
			T j = (target - vn) / wN;
			if (in.imB != T(0))
			{
				vb = madd(vb, j * in.imB, c.n);
				wb = madd(wb, j, p.jB[s]);
			}
			if (in.imA != T(0))
			{
				T mj = -j;
				va = madd(va, mj * in.imA, c.n);
				wa = madd(wa, mj, p.jA[s]);
			}
		}
		lambdaNTotal += lN > T(0) ? lN : T(0);
	}
	// rolling resistance, applied last: reverse first
	if (c.rolling > T(0) && lambdaNTotal > T(0))
	{
		V<T> wrel = sub(wb, wa);
		T wn = dot(wrel, c.n);
		V<T> wroll = sub(wrel, scale(wn, c.n));
		T wl = len(wroll);
		if (wl > T(1e-6))
		{
			T inv = T(1) / wl;
			V<T> axis = scale(inv, wroll);
			V<T> ya = mulv(in.iwA, axis), yb = mulv(in.iwB, axis);
			T kk = dot(axis, ya) + dot(axis, yb);
			if (kk > T(1e-12))
			{
				T maxDw = c.rolling * lambdaNTotal * invH * kk;
				bool takeMax = maxDw < wl;
				T dw = takeMax ? maxDw : wl;
				V<T> angImp = scale(dw / kk, axis);
				// wb' = wb - IwB angImp, wa' = wa + IwA angImp
				V<T> angImpb = vzero<T>();
				mulv_rev(in.iwB, angImp, neg(wbb), b.iwB, angImpb);
				mulv_rev(in.iwA, angImp, wab, b.iwA, angImpb);
				V<T> axisb = scale(dw / kk, angImpb);
				T sb = dot(angImpb, axis);
				T dwb = sb / kk;
				T kkb = -sb * dw / (kk * kk);
				T maxDwb = T(0), wlb = T(0);
				if (takeMax)
					maxDwb = dwb;
				else
					wlb = dwb;
				T lambdaTotb = maxDwb * c.rolling * invH * kk;
				kkb += maxDwb * c.rolling * lambdaNTotal * invH;
				axisb = madd(axisb, kkb, ya);
				axisb = madd(axisb, kkb, yb);
				mulv_rev(in.iwA, axis, scale(kkb, axis), b.iwA, axisb);
				mulv_rev(in.iwB, axis, scale(kkb, axis), b.iwB, axisb);
				V<T> wrollb = scale(inv, axisb);
				wlb += -dot(axisb, wroll) * inv * inv;
				len_rev(wroll, wl, wlb, wrollb);
				T nwr = dot(wrollb, c.n);
				V<T> wrelb = sub(wrollb, scale(nwr, c.n));
				cb.n = sub(cb.n, add(scale(wn, wrollb), scale(nwr, wrel)));
				wbb = add(wbb, wrelb);
				wab = sub(wab, wrelb);
				for (int s = 0; s < c.pointCount; ++s)
				{
					if (lambdaN[s] > T(0))
					{
						lambdaNb[s] += lambdaTotb;
					}
				}
			}
		}
	}
	for (int s = c.pointCount - 1; s >= 0; --s)
	{
		T lN = lambdaN[s];
		if (lN <= T(0))
		{
			continue;
		}
		va = sva[s];
		wa = swa[s];
		vb = svb[s];
		wb = swb[s];
		V<T> rAf, rBf;
		if (c.curved)
		{
			rAf = arm(c.shapeA, c.radiusA, in.qA, c.la[s], c.n, T(1));
			rBf = arm(c.shapeB, c.radiusB, in.qB, c.lb[s], c.n, T(-1));
		}
		else
		{
			rAf = p.rA[s];
			rBf = p.rB[s];
		}
		V<T> rAfb = vzero<T>(), rBfb = vzero<T>();
		// friction stage forward
		V<T> vrel = sub(add(vb, cross(wb, rBf)), add(va, cross(wa, rAf)));
		T vn = dot(vrel, c.n);
		V<T> vt = sub(vrel, scale(vn, c.n));
		T vtLen = len(vt);
		bool fric = false, takeStop = false, useMaxBranch = false;
		T wt = T(0), pStop = T(0), P = T(0);
		V<T> t = vzero<T>(), imp = vzero<T>();
		if (vtLen > T(1e-9))
		{
			t = scale(T(1) / vtLen, vt);
			wt = genInvMass(in.imA, in.iwA, rAf, t) + genInvMass(in.imB, in.iwB, rBf, t);
			if (wt > T(0))
			{
				fric = true;
				bool coherent = dot(t, c.slip[s]) > T(0.7);
				pStop = vtLen / wt;
				T pMax = c.mu * lN * invH;
				if (!coherent && vtLen < T(0.08))
				{
					takeStop = true;
				}
				else
				{
					takeStop = pStop < pMax;
					useMaxBranch = !takeStop;
				}
				P = takeStop ? pStop : pMax;
				imp = scale(-P, t);
			}
		}
		V<T> va1 = va, wa1 = wa, vb1 = vb, wb1 = wb;
		if (fric)
		{
			if (in.imB != T(0))
			{
				vb1 = madd(vb, in.imB, imp);
				wb1 = add(wb, mulv(in.iwB, cross(rBf, imp)));
			}
			if (in.imA != T(0))
			{
				V<T> pn = neg(imp);
				va1 = madd(va, in.imA, pn);
				wa1 = add(wa, mulv(in.iwA, cross(rAf, pn)));
			}
		}
		V<T> vrelPrev = sub(add(in.pvb, cross(in.pwb, rBf)), add(in.pva, cross(in.pwa, rAf)));
		T vnPrev = dot(vrelPrev, c.n);
		bool useE = dabs(vnPrev) > T(2) * in.gravityLen * in.h;
		T e = useE ? c.e : T(0);
		V<T> vrel2 = sub(add(vb1, cross(wb1, rBf)), add(va1, cross(wa1, rAf)));
		T vn2 = dot(vrel2, c.n);
		T target = -e * vnPrev;
		bool targetPos = target > T(0);
		target = targetPos ? target : T(0);
		T wN = p.wN[s];
		// normal impulse stage reverse
		V<T> va1b = vab, wa1b = wab, vb1b = vbb, wb1b = wbb;
		if (wN > T(0))
		{
			T j = (target - vn2) / wN;
			T jb = T(0);
			if (in.imB != T(0))
			{
				T d = dot(vbb, c.n);
				jb += in.imB * d + dot(wbb, p.jB[s]);
				b.imB += j * d;
				pb.jB[s] = madd(pb.jB[s], j, wbb);
				cb.n = madd(cb.n, j * in.imB, vbb);
			}
			if (in.imA != T(0))
			{
				T mj = -j;
				T d = dot(vab, c.n);
				T mjb = in.imA * d + dot(wab, p.jA[s]);
				b.imA += mj * d;
				pb.jA[s] = madd(pb.jA[s], mj, wab);
				cb.n = madd(cb.n, mj * in.imA, vab);
				jb -= mjb;
			}
			T targetb = jb / wN;
			T vn2b = -jb / wN;
			pb.wN[s] += -jb * j / wN;
			if (targetPos)
			{
				T eb = -targetb * vnPrev;
				T vnPrevb = -targetb * e;
				if (useE)
				{
					b.e += eb;
				}
				V<T> vrelPrevb = scale(vnPrevb, c.n);
				cb.n = madd(cb.n, vnPrevb, vrelPrev);
				b.pvb = add(b.pvb, vrelPrevb);
				cross_rev(in.pwb, rBf, vrelPrevb, b.pwb, rBfb);
				b.pva = sub(b.pva, vrelPrevb);
				cross_rev(in.pwa, rAf, neg(vrelPrevb), b.pwa, rAfb);
			}
			V<T> vrel2b = scale(vn2b, c.n);
			cb.n = madd(cb.n, vn2b, vrel2);
			vb1b = add(vb1b, vrel2b);
			cross_rev(wb1, rBf, vrel2b, wb1b, rBfb);
			va1b = sub(va1b, vrel2b);
			cross_rev(wa1, rAf, neg(vrel2b), wa1b, rAfb);
		}
		// friction stage reverse
		V<T> vab0 = va1b, wab0 = wa1b, vbb0 = vb1b, wbb0 = wb1b;
		if (fric)
		{
			V<T> impb = vzero<T>();
			if (in.imB != T(0))
			{
				impb = madd(impb, in.imB, vb1b);
				b.imB += dot(vb1b, imp);
				V<T> cB = cross(rBf, imp);
				V<T> cBb = vzero<T>();
				mulv_rev(in.iwB, cB, wb1b, b.iwB, cBb);
				cross_rev(rBf, imp, cBb, rBfb, impb);
			}
			if (in.imA != T(0))
			{
				V<T> pn = neg(imp);
				V<T> pnb = scale(in.imA, va1b);
				b.imA += dot(va1b, pn);
				V<T> cA = cross(rAf, pn);
				V<T> cAb = vzero<T>();
				mulv_rev(in.iwA, cA, wa1b, b.iwA, cAb);
				cross_rev(rAf, pn, cAb, rAfb, pnb);
				impb = sub(impb, pnb);
			}
			T Pb = -dot(impb, t);
			V<T> tb = scale(-P, impb);
			T pStopb = T(0);
			if (takeStop)
			{
				pStopb = Pb;
			}
			else if (useMaxBranch)
			{
				b.mu += Pb * lN * invH;
				lambdaNb[s] += Pb * c.mu * invH;
			}
			T vtLenb = pStopb / wt;
			T wtb = -pStopb * vtLen / (wt * wt);
			genInvMass_rev(in.iwA, rAf, t, wtb, b.imA, b.iwA, rAfb, tb);
			genInvMass_rev(in.iwB, rBf, t, wtb, b.imB, b.iwB, rBfb, tb);
			V<T> vtb = scale(T(1) / vtLen, tb);
			vtLenb += -dot(tb, vt) / (vtLen * vtLen);
			len_rev(vt, vtLen, vtLenb, vtb);
			T nvt = dot(vtb, c.n);
			V<T> vrelb = sub(vtb, scale(nvt, c.n));
			cb.n = sub(cb.n, add(scale(vn, vtb), scale(nvt, vrel)));
			vbb0 = add(vbb0, vrelb);
			cross_rev(wb, rBf, vrelb, wbb0, rBfb);
			vab0 = sub(vab0, vrelb);
			cross_rev(wa, rAf, neg(vrelb), wab0, rAfb);
		}
		vab = vab0;
		wab = wab0;
		vbb = vbb0;
		wbb = wbb0;
		// arms
		if (c.curved)
		{
			arm_rev(c.shapeA, c.radiusA, in.qA, c.la[s], T(1), rAfb, b.qA, cb.la[s], cb.n);
			arm_rev(c.shapeB, c.radiusB, in.qB, c.lb[s], T(-1), rBfb, b.qB, cb.lb[s], cb.n);
		}
		else
		{
			pb.rA[s] = add(pb.rA[s], rAfb);
			pb.rB[s] = add(pb.rB[s], rBfb);
		}
	}
}

} // namespace m3d_diff

#include "m3d_diff_gen.h"

namespace m3d_diff
{

// ---- one island through one recorded step ------------------------------------

// tape record of one contact in one substep (float, as stored on the device)
struct TapeContact
{
	int32_t a, b, pointCount, curved, shapeA, shapeB;
	float radiusA, radiusB;
	float n[3];
	float mu, e, rolling;
	float la[4][3], lb[4][3], off[4], fa[4][3], fb[4][3], slip[4][3];
	uint32_t id[4]; // feature ids of the points
	int32_t gen;    // kTapeGen* bits: how this substep's manifold came to be
};

// manifold generation events of a contact record
constexpr int32_t kTapeGenNarrow = 1;  // regenerated by the step's narrowphase at the step-start poses (substep 0)
constexpr int32_t kTapeGenPrepare = 2; // regenerated by this substep's contact preparation at the integrated poses
constexpr int32_t kTapeGenHeld = 4;    // held by the tunnelling guard (no generation)

// shape of a body, for manifold generation
struct TapeShape
{
	int32_t type;
	float radius;
	float he[3];
};

template <typename T>
M3D_DIFF_HD V<T> tv(const float* f)
{
	return v3<T>(T(f[0]), T(f[1]), T(f[2]));
}

template <typename T>
M3D_DIFF_HD Contact<T> loadContact(const TapeContact& t)
{
	Contact<T> c;
	c.a = t.a;
	c.b = t.b;
	c.pointCount = t.pointCount;
	c.curved = t.curved;
	c.shapeA = t.shapeA;
	c.shapeB = t.shapeB;
	c.radiusA = T(t.radiusA);
	c.radiusB = T(t.radiusB);
	c.n = tv<T>(t.n);
	c.mu = T(t.mu);
	c.e = T(t.e);
	c.rolling = T(t.rolling);
	for (int s = 0; s < 4; ++s)
	{
		c.la[s] = tv<T>(t.la[s]);
		c.lb[s] = tv<T>(t.lb[s]);
		c.off[s] = T(t.off[s]);
		c.fa[s] = tv<T>(t.fa[s]);
		c.fb[s] = tv<T>(t.fb[s]);
		c.slip[s] = tv<T>(t.slip[s]);
	}
	return c;
}

// island of one step: its bodies (global indices) and its contacts, in solve
// order, for each substep
struct TapeIsland
{
	int32_t bodyStart, bodyCount, contactStart, contactCount;
};

// per-operation inputs saved by the recording replay of a substep
template <typename T>
struct PoseRec
{
	V<T> pA, pB;
	Q<T> qA, qB;
	T lam[4];
	int gate;
	int reset; // points whose stiction anchors the pass re-seated at the local anchors
};
template <typename T>
struct VelRec
{
	V<T> va, wa, vb, wb;
};

// Everything the island driver reads and writes; body-indexed arrays are
// global (the island owns its dynamic bodies), contact-indexed arrays are
// indexed by the contact's position in the step's contact list.
template <typename T>
struct IslandCtx
{
	// constants
	const BodyConst<T>* bc;
	T h, invH, maxCorrection, gravityLen;
	V<T> g;
	int iterations, substeps;
	// the step
	const TapeIsland* island;
	const int32_t* bodies;        // the step's body list
	const TapeContact* contacts;  // [substep * contactsPerSubstep + position]
	int32_t contactsPerSubstep;
	// state: current (in/out), substep starts, integrated rotations and inverse
	// inertias, poses before reconstruction
	Body<T>* cur;
	Body<T>* start; // [substep * bodyCount + body]
	int32_t bodyCount;
	M<T>* iw;
	V<T>* x2;
	Q<T>* q2;
	// recording
	Prepared<T>* prep; // per position
	T* lamN;           // 4 per position
	T* lamT;
	PoseRec<T>* normRec; // [iteration * positions + position]
	PoseRec<T>* fricRec;
	VelRec<T>* velRec;
	int32_t positions;
	// adjoints
	Body<T>* adj;    // per body
	Body<T>* adj0;   // per body: adjoints of the substep start, accumulated
	T* imBar;        // per body: inverse mass
	T* ilBar;        // per body: isotropic inverse inertia
	T* muBar;        // per body: friction coefficient
	T* eBar;         // per body: restitution
	M<T>* iwBar;     // per body
	Prepared<T>* prepBar;
	T* lamNBar;      // 4 per position
	T* lamTBar;
	const T* muBody; // per body friction and restitution (to split contact values)
	const T* eBody;
	// manifold data as state
	ContactBar<T>* cbar;             // per position: adjoint of the contact's manifold data
	const TapeShape* shapes;         // per body
	const TapeContact* prevContacts; // the previous step's records (its last substep), or null
	const int32_t* prevPos;          // per position: the contact's position in the previous step, or -1
	T dt;                            // step length (narrowphase margin)
	const double* genJ;              // per position: the narrowphase generation's Jacobian, or null (computed here)
	// regenerating replay (verification): when set, the manifolds are state
	// carried here and regenerated at the recorded generation events instead
	// of read from the tape
	Contact<T>* live;
	uint32_t* liveIds; // 4 per position
	// the team working the island: one thread (lane 0 of width 1, order null),
	// or a warp whose lanes take the contacts of one dependency level at a
	// time (see ContactRun)
	int lane, width;
	const int32_t* order;      // per position of the island: its positions by level, or null
	const int32_t* orderLevel; // the level of each entry of order
};

// ---- island teams -----------------------------------------------------------------
// A contact's dependency level is one above the latest earlier contact of its
// island that shares a dynamic body with it (static bodies are only read).
// The contacts of one level touch disjoint dynamic bodies, and every body
// meets its contacts in the recorded order when the levels are walked upwards
// (forward passes) or downwards (reverse passes): lanes may take one level's
// contacts at once and the result is bitwise that of one thread walking the
// recorded order.  A run is up to `width` contacts of one level; after each
// run the team synchronises.
struct ContactRun
{
	int j, pos, count;
	bool mine, more, rev;
};

template <typename T>
M3D_DIFF_HD void teamSync(const IslandCtx<T>& x)
{
#ifdef __CUDA_ARCH__
	if (x.width > 1)
	{
		__syncwarp();
	}
#endif
}

template <typename T>
M3D_DIFF_HD void contactRunSetup(const IslandCtx<T>& x, const TapeIsland& r, ContactRun& u)
{
	const int n = r.contactCount;
	u.more = u.rev ? u.j > 0 : u.j < n;
	u.count = 1;
	u.mine = u.more;
	u.pos = r.contactStart + (u.rev ? u.j - 1 : u.j);
#ifdef __CUDA_ARCH__
	if (x.order != nullptr && u.more)
	{
		const int head = u.rev ? u.j - 1 : u.j;
		const int level = x.orderLevel[r.contactStart + head];
		const int idx = u.rev ? u.j - 1 - x.lane : u.j + x.lane;
		u.mine = idx >= 0 && idx < n && x.orderLevel[r.contactStart + idx] == level;
		u.pos = u.mine ? x.order[r.contactStart + idx] : -1;
		u.count = __popc(__ballot_sync(0xffffffffu, u.mine));
	}
#endif
}

// the first run of the island's contacts, upwards (rev false) or downwards
template <typename T>
M3D_DIFF_HD ContactRun contactRunBegin(const IslandCtx<T>& x, const TapeIsland& r, bool rev)
{
	ContactRun u;
	u.rev = rev;
	u.j = rev ? r.contactCount : 0;
	contactRunSetup(x, r, u);
	return u;
}

template <typename T>
M3D_DIFF_HD void contactRunNext(const IslandCtx<T>& x, const TapeIsland& r, ContactRun& u)
{
	teamSync(x);
	u.j += u.rev ? -u.count : u.count;
	contactRunSetup(x, r, u);
}

template <typename T>
M3D_DIFF_HD Contact<T> contactOf(const IslandCtx<T>& x, const TapeContact* tc, int pos)
{
	return x.live != nullptr ? x.live[pos] : loadContact<T>(tc[pos]);
}

template <typename T>
M3D_DIFF_HD void regenerateLive(const IslandCtx<T>& x, const TapeContact& rec, int pos, V<T> xA, Q<T> qA, V<T> xB,
								Q<T> qB, T margin);

template <typename T>
M3D_DIFF_HD_CALL void substepForward(const IslandCtx<T>& x, const TapeIsland& r, int sub, bool record)
{
	const BodyConst<T>* bc = x.bc;
	for (int k = x.lane; k < r.bodyCount; k += x.width)
	{
		int i = x.bodies[r.bodyStart + k];
		if (!bc[i].dynamic)
		{
			continue;
		}
		Body<T> s1;
		integrate(x.cur[i], bc[i], x.h, x.g, s1, x.iw[i]);
		x.start[(size_t)sub * x.bodyCount + i] = x.cur[i];
		x.cur[i] = s1;
	}
	teamSync(x);
	const TapeContact* tc = x.contacts + (size_t)sub * x.contactsPerSubstep;
	if (x.live != nullptr)
	{
		for (int j = 0; j < r.contactCount; ++j)
		{
			const int pos = r.contactStart + j;
			if (tc[pos].gen & kTapeGenPrepare)
			{
				const Body<T>& A = x.cur[tc[pos].a];
				const Body<T>& B = x.cur[tc[pos].b];
				regenerateLive(x, tc[pos], pos, A.x, A.q, B.x, B.q,
							   T(kGenSpeculativeBase) + x.h * len(m3d_diff::sub(A.v, B.v)));
			}
			// slip directions only steer branches: as the engine had them
			for (int q = 0; q < 4; ++q)
			{
				x.live[pos].slip[q] = tv<T>(tc[pos].slip[q]);
			}
		}
	}
	for (int j = x.lane; j < r.contactCount; j += x.width)
	{
		int pos = r.contactStart + j;
		Contact<T> c = contactOf(x, tc, pos);
		Prepared<T>& p = x.prep[pos];
		preparedZero(p);
		prepare(c, x.cur[c.a].q, x.cur[c.b].q, bc[c.a].invMass, bc[c.b].invMass, x.iw[c.a], x.iw[c.b], p);
		for (int s = 0; s < 4; ++s)
		{
			x.lamN[4 * pos + s] = T(0);
			x.lamT[4 * pos + s] = T(0);
		}
	}
	teamSync(x);
	for (int it = 0; it < x.iterations; ++it)
	{
		for (ContactRun u = contactRunBegin(x, r, false); u.more; contactRunNext(x, r, u))
		{
			if (!u.mine)
			{
				continue;
			}
			const int pos = u.pos;
			Contact<T> c = contactOf(x, tc, pos);
			if (record)
			{
				PoseRec<T>& rec = x.normRec[(size_t)it * x.positions + pos];
				rec.pA = x.cur[c.a].x;
				rec.qA = x.cur[c.a].q;
				rec.pB = x.cur[c.b].x;
				rec.qB = x.cur[c.b].q;
			}
			if (c.pointCount == 0)
			{
				continue;
			}
			normals(c, x.prep[pos], bc[c.a].invMass, bc[c.b].invMass, x.maxCorrection, x.cur[c.a].x, x.cur[c.a].q,
					x.cur[c.b].x, x.cur[c.b].q, x.lamN + 4 * pos);
		}
	}
	for (ContactRun u = contactRunBegin(x, r, false); u.more; contactRunNext(x, r, u))
	{
		if (!u.mine)
		{
			continue;
		}
		const int pos = u.pos;
		Contact<T> c = contactOf(x, tc, pos);
		bool gate = frictionGate(c, x.prep[pos], x.cur[c.a].v, x.cur[c.a].w, x.cur[c.b].v, x.cur[c.b].w);
		if (record)
		{
			PoseRec<T>& rec = x.fricRec[pos];
			rec.pA = x.cur[c.a].x;
			rec.qA = x.cur[c.a].q;
			rec.pB = x.cur[c.b].x;
			rec.qB = x.cur[c.b].q;
			for (int s = 0; s < 4; ++s)
			{
				rec.lam[s] = x.lamT[4 * pos + s];
			}
			rec.gate = gate ? 1 : 0;
		}
		// a sliding box-box contact re-seats all its anchors instead
		int reset = c.shapeA == kShapeBox && c.shapeB == kShapeBox && c.pointCount > 0 && !gate
						? (1 << c.pointCount) - 1
						: 0;
		if (gate)
		{
			friction(c, bc[c.a].invMass, bc[c.b].invMass, x.iw[c.a], x.iw[c.b], x.lamN + 4 * pos, x.cur[c.a].x,
					 x.cur[c.a].q, x.cur[c.b].x, x.cur[c.b].q, x.lamT + 4 * pos, &reset);
		}
		if (record)
		{
			x.fricRec[pos].reset = reset;
		}
		if (x.live != nullptr)
		{
			for (int q = 0; q < 4; ++q)
			{
				if ((reset >> q) & 1)
				{
					x.live[pos].fa[q] = x.live[pos].la[q];
					x.live[pos].fb[q] = x.live[pos].lb[q];
				}
			}
		}
	}
	for (int k = x.lane; k < r.bodyCount; k += x.width)
	{
		int i = x.bodies[r.bodyStart + k];
		if (!bc[i].dynamic)
		{
			continue;
		}
		const Body<T>& s0 = x.start[(size_t)sub * x.bodyCount + i];
		x.x2[i] = x.cur[i].x;
		x.q2[i] = x.cur[i].q;
		reconstruct(x.cur[i].x, x.cur[i].q, s0.x, s0.q, x.invH, x.cur[i].v, x.cur[i].w);
	}
	teamSync(x);
	for (ContactRun u = contactRunBegin(x, r, false); u.more; contactRunNext(x, r, u))
	{
		if (!u.mine)
		{
			continue;
		}
		const int pos = u.pos;
		Contact<T> c = contactOf(x, tc, pos);
		if (record)
		{
			VelRec<T>& rec = x.velRec[pos];
			rec.va = x.cur[c.a].v;
			rec.wa = x.cur[c.a].w;
			rec.vb = x.cur[c.b].v;
			rec.wb = x.cur[c.b].w;
		}
		VelocityIn<T> in;
		in.imA = bc[c.a].invMass;
		in.imB = bc[c.b].invMass;
		in.iwA = x.iw[c.a];
		in.iwB = x.iw[c.b];
		in.qA = x.cur[c.a].q;
		in.qB = x.cur[c.b].q;
		const Body<T>& sa = x.start[(size_t)sub * x.bodyCount + c.a];
		const Body<T>& sb = x.start[(size_t)sub * x.bodyCount + c.b];
		in.pva = bc[c.a].dynamic ? sa.v : x.cur[c.a].v;
		in.pwa = bc[c.a].dynamic ? sa.w : x.cur[c.a].w;
		in.pvb = bc[c.b].dynamic ? sb.v : x.cur[c.b].v;
		in.pwb = bc[c.b].dynamic ? sb.w : x.cur[c.b].w;
		in.h = x.h;
		in.gravityLen = x.gravityLen;
		V<T> va = x.cur[c.a].v, wa = x.cur[c.a].w, vb = x.cur[c.b].v, wb = x.cur[c.b].w;
		velocity(c, x.prep[pos], in, x.lamN + 4 * pos, va, wa, vb, wb);
		if (bc[c.a].dynamic)
		{
			x.cur[c.a].v = va;
			x.cur[c.a].w = wa;
		}
		if (bc[c.b].dynamic)
		{
			x.cur[c.b].v = vb;
			x.cur[c.b].w = wb;
		}
	}
}

// friction coefficient of a contact: sqrt(mu_a mu_b); adjoint split
template <typename T>
M3D_DIFF_HD void scatterMaterials(const IslandCtx<T>& x, const Contact<T>& c, T muB, T eB)
{
	const T ma = x.muBody[c.a], mb = x.muBody[c.b];
	if (x.bc[c.a].dynamic && ma > T(0))
	{
		x.muBar[c.a] += muB * T(0.5) * c.mu / ma;
	}
	if (x.bc[c.b].dynamic && mb > T(0))
	{
		x.muBar[c.b] += muB * T(0.5) * c.mu / mb;
	}
	// restitution: the larger of the two, B's on ties, as contact creation
	// picks it (reference src/world.cpp:1540-1568)
	const int who = x.eBody[c.a] > x.eBody[c.b] ? c.a : c.b;
	if (x.bc[who].dynamic)
	{
		x.eBar[who] += eB;
	}
}

// ---- manifold generation events ---------------------------------------------------

// Jacobian of a manifold generation (reference src/collide.cpp:813-859 with
// the offsets of src/world.cpp:1738-1845) with respect to the generation
// poses: J[o * kGenJCols + k], rows o = the normal (3), then per recorded
// point i (up to 4, matched to the generated points by feature id) its local
// anchors on A (3) and B (3) and its separation offset (1); columns k = A's
// position and rotation (0..6), then B's (7..13).  Forward-mode dual numbers
// carry only the seeded (dynamic) bodies' columns: N = 7 or 14.  Rows of an
// unmatched point, and all rows when the generated normal is not the
// recorded one, are zero.
constexpr int kGenJRows = 31;
constexpr int kGenJCols = 14;

template <typename T, int N>
M3D_DIFF_HD_CALL void generationJacobianN(const TapeShape& shA, const TapeShape& shB, const TapeContact& rec, V<T> xA,
										  Q<T> qA, V<T> xB, Q<T> qB, T margin, bool seedA, bool seedB, double* J)
{
	typedef Dual<T, N> S;
	for (int o = 0; o < kGenJRows * kGenJCols; ++o)
	{
		J[o] = 0.0;
	}
	GenShape<S> sa, sb;
	sa.type = shA.type;
	sa.radius = S(T(shA.radius));
	sa.he = v3<S>(S(T(shA.he[0])), S(T(shA.he[1])), S(T(shA.he[2])));
	sb.type = shB.type;
	sb.radius = S(T(shB.radius));
	sb.he = v3<S>(S(T(shB.he[0])), S(T(shB.he[1])), S(T(shB.he[2])));
	// dual slots: A's pose first when A is seeded, then B's
	const int oA = 0, oB = seedA ? 7 : 0;
	V<S> gxA = v3<S>(S(xA.x), S(xA.y), S(xA.z));
	Q<S> gqA = q4<S>(S(qA.x), S(qA.y), S(qA.z), S(qA.w));
	V<S> gxB = v3<S>(S(xB.x), S(xB.y), S(xB.z));
	Q<S> gqB = q4<S>(S(qB.x), S(qB.y), S(qB.z), S(qB.w));
	if (seedA)
	{
		gxA.x.d[oA + 0] = gxA.y.d[oA + 1] = gxA.z.d[oA + 2] = 1.0;
		gqA.x.d[oA + 3] = gqA.y.d[oA + 4] = gqA.z.d[oA + 5] = gqA.w.d[oA + 6] = 1.0;
	}
	if (seedB)
	{
		gxB.x.d[oB + 0] = gxB.y.d[oB + 1] = gxB.z.d[oB + 2] = 1.0;
		gqB.x.d[oB + 3] = gqB.y.d[oB + 4] = gqB.z.d[oB + 5] = gqB.w.d[oB + 6] = 1.0;
	}
	GenManifold<S> g;
	genManifold(sa, gxA, gqA, sb, gxB, gqB, S(margin), g);
	const bool sameNormal =
		g.count > 0 && g.n.x.v * T(rec.n[0]) + g.n.y.v * T(rec.n[1]) + g.n.z.v * T(rec.n[2]) > T(0.999);
	if (!sameNormal)
	{
		return;
	}
	// dual slot k -> Jacobian column
	int col[N];
	for (int k = 0; k < N; ++k)
	{
		col[k] = (seedA && k < 7) ? k : 7 + (k - oB);
	}
	for (int k = 0; k < N; ++k)
	{
		J[0 * kGenJCols + col[k]] = g.n.x.d[k];
		J[1 * kGenJCols + col[k]] = g.n.y.d[k];
		J[2 * kGenJCols + col[k]] = g.n.z.d[k];
	}
	for (int i = 0; i < rec.pointCount; ++i)
	{
		int j = -1;
		for (int q = 0; q < g.count; ++q)
		{
			if (g.p[q].id == rec.id[i])
			{
				j = q;
				break;
			}
		}
		if (j < 0)
		{
			continue;
		}
		const GenPoint<S>& gp = g.p[j];
		double* r = J + (3 + 7 * i) * kGenJCols;
		for (int k = 0; k < N; ++k)
		{
			r[0 * kGenJCols + col[k]] = gp.la.x.d[k];
			r[1 * kGenJCols + col[k]] = gp.la.y.d[k];
			r[2 * kGenJCols + col[k]] = gp.la.z.d[k];
			r[3 * kGenJCols + col[k]] = gp.lb.x.d[k];
			r[4 * kGenJCols + col[k]] = gp.lb.y.d[k];
			r[5 * kGenJCols + col[k]] = gp.lb.z.d[k];
			r[6 * kGenJCols + col[k]] = gp.off.d[k];
		}
	}
}

// Columns p and p + 7 of the same Jacobian (component p of A's and of B's
// pose: x, y, z, qx, qy, qz, qw), two dual slots wide, so that seven threads
// share one generation.  Forward-mode lanes do not mix, so each column equals
// the one generationJacobian gives; a column of a non-dynamic body is zero.
template <typename T>
M3D_DIFF_HD_CALL void generationJacobianPair(const BodyConst<T>* bc, const TapeShape* shapes, const TapeContact& rec,
											 V<T> xA, Q<T> qA, V<T> xB, Q<T> qB, T margin, int p, double* J)
{
	typedef Dual<T, 2> S;
	const int cA = p, cB = 7 + p;
	for (int o = 0; o < kGenJRows; ++o)
	{
		J[o * kGenJCols + cA] = 0.0;
		J[o * kGenJCols + cB] = 0.0;
	}
	const bool dynA = bc[rec.a].dynamic != 0, dynB = bc[rec.b].dynamic != 0;
	if ((!dynA && !dynB) || rec.pointCount == 0)
	{
		return;
	}
	const TapeShape& shA = shapes[rec.a];
	const TapeShape& shB = shapes[rec.b];
	GenShape<S> sa, sb;
	sa.type = shA.type;
	sa.radius = S(T(shA.radius));
	sa.he = v3<S>(S(T(shA.he[0])), S(T(shA.he[1])), S(T(shA.he[2])));
	sb.type = shB.type;
	sb.radius = S(T(shB.radius));
	sb.he = v3<S>(S(T(shB.he[0])), S(T(shB.he[1])), S(T(shB.he[2])));
	V<S> gxA = v3<S>(S(xA.x), S(xA.y), S(xA.z));
	Q<S> gqA = q4<S>(S(qA.x), S(qA.y), S(qA.z), S(qA.w));
	V<S> gxB = v3<S>(S(xB.x), S(xB.y), S(xB.z));
	Q<S> gqB = q4<S>(S(qB.x), S(qB.y), S(qB.z), S(qB.w));
	S* inA[7] = { &gxA.x, &gxA.y, &gxA.z, &gqA.x, &gqA.y, &gqA.z, &gqA.w };
	S* inB[7] = { &gxB.x, &gxB.y, &gxB.z, &gqB.x, &gqB.y, &gqB.z, &gqB.w };
	if (dynA)
	{
		inA[p]->d[0] = 1.0;
	}
	if (dynB)
	{
		inB[p]->d[1] = 1.0;
	}
	GenManifold<S> g;
	genManifold(sa, gxA, gqA, sb, gxB, gqB, S(margin), g);
	const bool sameNormal =
		g.count > 0 && g.n.x.v * T(rec.n[0]) + g.n.y.v * T(rec.n[1]) + g.n.z.v * T(rec.n[2]) > T(0.999);
	if (!sameNormal)
	{
		return;
	}
	const int col[2] = { cA, cB };
	const bool live[2] = { dynA, dynB };
	for (int k = 0; k < 2; ++k)
	{
		if (!live[k])
		{
			continue;
		}
		J[0 * kGenJCols + col[k]] = g.n.x.d[k];
		J[1 * kGenJCols + col[k]] = g.n.y.d[k];
		J[2 * kGenJCols + col[k]] = g.n.z.d[k];
	}
	for (int i = 0; i < rec.pointCount; ++i)
	{
		int j = -1;
		for (int q = 0; q < g.count; ++q)
		{
			if (g.p[q].id == rec.id[i])
			{
				j = q;
				break;
			}
		}
		if (j < 0)
		{
			continue;
		}
		const GenPoint<S>& gp = g.p[j];
		double* r = J + (3 + 7 * i) * kGenJCols;
		for (int k = 0; k < 2; ++k)
		{
			if (!live[k])
			{
				continue;
			}
			r[0 * kGenJCols + col[k]] = gp.la.x.d[k];
			r[1 * kGenJCols + col[k]] = gp.la.y.d[k];
			r[2 * kGenJCols + col[k]] = gp.la.z.d[k];
			r[3 * kGenJCols + col[k]] = gp.lb.x.d[k];
			r[4 * kGenJCols + col[k]] = gp.lb.y.d[k];
			r[5 * kGenJCols + col[k]] = gp.lb.z.d[k];
			r[6 * kGenJCols + col[k]] = gp.off.d[k];
		}
	}
}

// the Jacobian of the contact's generation, for its dynamic bodies
template <typename T>
M3D_DIFF_HD void generationJacobian(const BodyConst<T>* bc, const TapeShape* shapes, const TapeContact& rec, V<T> xA,
									Q<T> qA, V<T> xB, Q<T> qB, T margin, double* J)
{
	const bool dynA = bc[rec.a].dynamic != 0, dynB = bc[rec.b].dynamic != 0;
	if ((!dynA && !dynB) || rec.pointCount == 0)
	{
		for (int o = 0; o < kGenJRows * kGenJCols; ++o)
		{
			J[o] = 0.0;
		}
		return;
	}
	if (dynA && dynB)
	{
		generationJacobianN<T, 14>(shapes[rec.a], shapes[rec.b], rec, xA, qA, xB, qB, margin, true, true, J);
	}
	else
	{
		generationJacobianN<T, 7>(shapes[rec.a], shapes[rec.b], rec, xA, qA, xB, qB, margin, dynA, dynB, J);
	}
}

// Adds J^T (adjoint of the manifold data) to the pose adjoints of the
// contact's dynamic bodies, summed in double.
template <typename T>
M3D_DIFF_HD void applyGenerationJacobian(const IslandCtx<T>& x, const TapeContact& rec, const double* J,
										 const ContactBar<T>& cb)
{
	T bar[kGenJRows];
	bar[0] = cb.n.x;
	bar[1] = cb.n.y;
	bar[2] = cb.n.z;
	for (int i = 0; i < 4; ++i)
	{
		const bool on = i < rec.pointCount;
		T* r = bar + 3 + 7 * i;
		r[0] = on ? cb.la[i].x : T(0);
		r[1] = on ? cb.la[i].y : T(0);
		r[2] = on ? cb.la[i].z : T(0);
		r[3] = on ? cb.lb[i].x : T(0);
		r[4] = on ? cb.lb[i].y : T(0);
		r[5] = on ? cb.lb[i].z : T(0);
		r[6] = on ? cb.off[i] : T(0);
	}
	double acc[kGenJCols];
	for (int k = 0; k < kGenJCols; ++k)
	{
		acc[k] = 0.0;
	}
	for (int o = 0; o < kGenJRows; ++o)
	{
		if (bar[o] == T(0))
		{
			continue;
		}
		for (int k = 0; k < kGenJCols; ++k)
		{
			// a zero entry carries nothing (not even an infinite adjoint's NaN)
			const double j = J[o * kGenJCols + k];
			if (j != 0.0)
			{
				acc[k] += (double)bar[o] * j;
			}
		}
	}
	if (x.bc[rec.a].dynamic)
	{
		x.adj[rec.a].x = add(x.adj[rec.a].x, v3<T>(T(acc[0]), T(acc[1]), T(acc[2])));
		x.adj[rec.a].q = qadd(x.adj[rec.a].q, q4<T>(T(acc[3]), T(acc[4]), T(acc[5]), T(acc[6])));
	}
	if (x.bc[rec.b].dynamic)
	{
		x.adj[rec.b].x = add(x.adj[rec.b].x, v3<T>(T(acc[7]), T(acc[8]), T(acc[9])));
		x.adj[rec.b].q = qadd(x.adj[rec.b].q, q4<T>(T(acc[10]), T(acc[11]), T(acc[12]), T(acc[13])));
	}
}

// the adjoint of a generation computed on the spot
template <typename T>
M3D_DIFF_HD_CALL void generationAdjoint(const IslandCtx<T>& x, const TapeContact& rec, V<T> xA, Q<T> qA, V<T> xB,
										Q<T> qB, T margin, const ContactBar<T>& cb)
{
	double J[kGenJRows * kGenJCols];
	generationJacobian(x.bc, x.shapes, rec, xA, qA, xB, qB, margin, J);
	applyGenerationJacobian(x, rec, J, cb);
}

// The stiction anchors a generated manifold starts with are fresh (equal to
// its local anchors) or kept from the old point with the same feature id.
// Moves the anchor adjoints of cb accordingly: fresh ones onto the local
// anchors, kept ones into cbOld (the adjoint of the old manifold, whose point
// order oldIds gives; null: the old manifold is not on the tape and kept
// anchors count as constants).  cb's anchor adjoints end at zero.
template <typename T>
M3D_DIFF_HD void generationAnchors(const TapeContact& rec, const uint32_t* oldIds, int oldCount, ContactBar<T>& cb,
								   ContactBar<T>& cbOld)
{
	contactBarZero(cbOld);
	for (int i = 0; i < rec.pointCount; ++i)
	{
		bool fresh = true;
		for (int k = 0; k < 3; ++k)
		{
			fresh = fresh && rec.fa[i][k] == rec.la[i][k] && rec.fb[i][k] == rec.lb[i][k];
		}
		if (fresh)
		{
			cb.la[i] = add(cb.la[i], cb.fa[i]);
			cb.lb[i] = add(cb.lb[i], cb.fb[i]);
		}
		else if (oldIds != nullptr)
		{
			for (int j = 0; j < oldCount; ++j)
			{
				if (oldIds[j] == rec.id[i])
				{
					cbOld.fa[j] = add(cbOld.fa[j], cb.fa[i]);
					cbOld.fb[j] = add(cbOld.fb[j], cb.fb[i]);
					break;
				}
			}
		}
		cb.fa[i] = vzero<T>();
		cb.fb[i] = vzero<T>();
	}
}

// A generation event of a contact: anchors, then the Jacobian at the
// generation poses; cb becomes the old manifold's adjoint.
template <typename T>
M3D_DIFF_HD void reverseGeneration(const IslandCtx<T>& x, const TapeContact& rec, const TapeContact* old, V<T> xA,
								   Q<T> qA, V<T> xB, Q<T> qB, T margin, ContactBar<T>& cb, const double* J = nullptr)
{
	ContactBar<T> cbOld;
	generationAnchors(rec, old != nullptr ? old->id : nullptr, old != nullptr ? old->pointCount : 0, cb, cbOld);
	if (J != nullptr)
	{
		applyGenerationJacobian(x, rec, J, cb);
	}
	else
	{
		generationAdjoint(x, rec, xA, qA, xB, qB, margin, cb);
	}
	cb = cbOld;
}

// Regeneration of a live manifold (regenerating replay): the engine's
// collision at the given poses, then the inheritance of slip directions and,
// box-box only, of stiction anchors that have neither slipped nor drifted
// from the old manifold (reference src/collide.cpp:865-913).
template <typename T>
M3D_DIFF_HD void regenerateLive(const IslandCtx<T>& x, const TapeContact& rec, int pos, V<T> xA, Q<T> qA, V<T> xB,
								Q<T> qB, T margin)
{
	Contact<T>& c = x.live[pos];
	uint32_t* ids = x.liveIds + 4 * pos;
	const Contact<T> old = c;
	const uint32_t oldIds[4] = { ids[0], ids[1], ids[2], ids[3] };
	GenShape<T> sa, sb;
	sa.type = x.shapes[rec.a].type;
	sa.radius = T(x.shapes[rec.a].radius);
	sa.he = v3<T>(T(x.shapes[rec.a].he[0]), T(x.shapes[rec.a].he[1]), T(x.shapes[rec.a].he[2]));
	sb.type = x.shapes[rec.b].type;
	sb.radius = T(x.shapes[rec.b].radius);
	sb.he = v3<T>(T(x.shapes[rec.b].he[0]), T(x.shapes[rec.b].he[1]), T(x.shapes[rec.b].he[2]));
	GenManifold<T> g;
	genManifold(sa, xA, qA, sb, xB, qB, margin, g);
	const bool boxBox = sa.type == kShapeBox && sb.type == kShapeBox;
	c.pointCount = g.count;
	c.n = g.n;
	for (int i = 0; i < g.count; ++i)
	{
		c.la[i] = g.p[i].la;
		c.lb[i] = g.p[i].lb;
		c.off[i] = g.p[i].off;
		c.fa[i] = c.la[i];
		c.fb[i] = c.lb[i];
		c.slip[i] = vzero<T>();
		ids[i] = g.p[i].id;
		for (int j = 0; j < old.pointCount; ++j)
		{
			if (oldIds[j] != ids[i])
			{
				continue;
			}
			c.slip[i] = old.slip[j];
			if (!boxBox)
			{
				break;
			}
			V<T> pAold = add(rotate(qA, old.fa[j]), xA);
			V<T> pBold = add(rotate(qB, old.fb[j]), xB);
			V<T> pAnew = add(rotate(qA, c.la[i]), xA);
			V<T> gap = sub(pBold, pAold);
			V<T> dpt = sub(gap, scale(dot(gap, c.n), c.n));
			V<T> drift = sub(pAold, pAnew);
			if (dot(dpt, dpt) < T(0.02f * 0.02f) && dot(drift, drift) < T(0.05f * 0.05f))
			{
				c.fa[i] = old.fa[j];
				c.fb[i] = old.fb[j];
			}
			break;
		}
	}
}

// the record of a contact before the step (its previous step's last substep), or null
template <typename T>
M3D_DIFF_HD const TapeContact* previousRecord(const IslandCtx<T>& x, int pos)
{
	if (x.prevContacts == nullptr || x.prevPos == nullptr || x.prevPos[pos] < 0)
	{
		return nullptr;
	}
	return x.prevContacts + x.prevPos[pos];
}

template <typename T>
M3D_DIFF_HD_CALL void substepReverse(const IslandCtx<T>& x, const TapeIsland& r, int sub)
{
	const BodyConst<T>* bc = x.bc;
	const TapeContact* tc = x.contacts + (size_t)sub * x.contactsPerSubstep;
	for (int k = x.lane; k < r.bodyCount; k += x.width)
	{
		int i = x.bodies[r.bodyStart + k];
		x.adj0[i] = bodyZero<T>();
		M<T> z;
		z.cx = z.cy = z.cz = vzero<T>();
		x.iwBar[i] = z;
	}
	teamSync(x);
	for (int j = x.lane; j < r.contactCount; j += x.width)
	{
		int pos = r.contactStart + j;
		preparedZero(x.prepBar[pos]);
		for (int s = 0; s < 4; ++s)
		{
			x.lamNBar[4 * pos + s] = T(0);
			x.lamTBar[4 * pos + s] = T(0);
		}
	}
	teamSync(x);
	// velocity pass, in reverse contact order
	for (ContactRun u = contactRunBegin(x, r, true); u.more; contactRunNext(x, r, u))
	{
		if (!u.mine)
		{
			continue;
		}
		const int pos = u.pos;
		Contact<T> c = loadContact<T>(tc[pos]);
		const VelRec<T>& rec = x.velRec[pos];
		VelocityIn<T> in;
		in.imA = bc[c.a].invMass;
		in.imB = bc[c.b].invMass;
		in.iwA = x.iw[c.a];
		in.iwB = x.iw[c.b];
		in.qA = x.x2 != nullptr && bc[c.a].dynamic ? x.q2[c.a] : x.cur[c.a].q;
		in.qB = x.x2 != nullptr && bc[c.b].dynamic ? x.q2[c.b] : x.cur[c.b].q;
		const Body<T>& sa = x.start[(size_t)sub * x.bodyCount + c.a];
		const Body<T>& sb = x.start[(size_t)sub * x.bodyCount + c.b];
		in.pva = bc[c.a].dynamic ? sa.v : x.cur[c.a].v;
		in.pwa = bc[c.a].dynamic ? sa.w : x.cur[c.a].w;
		in.pvb = bc[c.b].dynamic ? sb.v : x.cur[c.b].v;
		in.pwb = bc[c.b].dynamic ? sb.w : x.cur[c.b].w;
		in.h = x.h;
		in.gravityLen = x.gravityLen;
		VelocityBar<T> b;
		b.imA = b.imB = b.mu = b.e = T(0);
		b.iwA.cx = b.iwA.cy = b.iwA.cz = vzero<T>();
		b.iwB = b.iwA;
		b.qA = b.qB = qzero<T>();
		b.pva = b.pwa = b.pvb = b.pwb = vzero<T>();
		V<T> dummy0 = vzero<T>(), dummy1 = vzero<T>(), dummy2 = vzero<T>(), dummy3 = vzero<T>();
		V<T>& vab = bc[c.a].dynamic ? x.adj[c.a].v : dummy0;
		V<T>& wab = bc[c.a].dynamic ? x.adj[c.a].w : dummy1;
		V<T>& vbb = bc[c.b].dynamic ? x.adj[c.b].v : dummy2;
		V<T>& wbb = bc[c.b].dynamic ? x.adj[c.b].w : dummy3;
		velocity_rev(c, x.prep[pos], in, x.lamN + 4 * pos, rec.va, rec.wa, rec.vb, rec.wb, vab, wab, vbb, wbb,
					 x.prepBar[pos], x.lamNBar + 4 * pos, b, x.cbar[pos]);
		if (bc[c.a].dynamic)
		{
			x.imBar[c.a] += b.imA;
			x.iwBar[c.a].cx = add(x.iwBar[c.a].cx, b.iwA.cx);
			x.iwBar[c.a].cy = add(x.iwBar[c.a].cy, b.iwA.cy);
			x.iwBar[c.a].cz = add(x.iwBar[c.a].cz, b.iwA.cz);
			x.adj[c.a].q = qadd(x.adj[c.a].q, b.qA);
			x.adj0[c.a].v = add(x.adj0[c.a].v, b.pva);
			x.adj0[c.a].w = add(x.adj0[c.a].w, b.pwa);
		}
		if (bc[c.b].dynamic)
		{
			x.imBar[c.b] += b.imB;
			x.iwBar[c.b].cx = add(x.iwBar[c.b].cx, b.iwB.cx);
			x.iwBar[c.b].cy = add(x.iwBar[c.b].cy, b.iwB.cy);
			x.iwBar[c.b].cz = add(x.iwBar[c.b].cz, b.iwB.cz);
			x.adj[c.b].q = qadd(x.adj[c.b].q, b.qB);
			x.adj0[c.b].v = add(x.adj0[c.b].v, b.pvb);
			x.adj0[c.b].w = add(x.adj0[c.b].w, b.pwb);
		}
		scatterMaterials(x, c, b.mu, b.e);
	}
	// reconstruction
	for (int k = x.lane; k < r.bodyCount; k += x.width)
	{
		int i = x.bodies[r.bodyStart + k];
		if (!bc[i].dynamic)
		{
			continue;
		}
		const Body<T>& s0 = x.start[(size_t)sub * x.bodyCount + i];
		V<T> vb = x.adj[i].v, wb = x.adj[i].w;
		x.adj[i].v = vzero<T>();
		x.adj[i].w = vzero<T>();
		reconstruct_rev(x.x2[i], x.q2[i], s0.x, s0.q, x.invH, vb, wb, x.adj[i].x, x.adj[i].q, x.adj0[i].x, x.adj0[i].q);
	}
	teamSync(x);
	// friction, reverse contact order
	for (ContactRun u = contactRunBegin(x, r, true); u.more; contactRunNext(x, r, u))
	{
		if (!u.mine)
		{
			continue;
		}
		const int pos = u.pos;
		const PoseRec<T>& rec = x.fricRec[pos];
		ContactBar<T>& cb = x.cbar[pos];
		for (int s = 0; s < 4; ++s)
		{
			if ((rec.reset >> s) & 1)
			{
				// re-seated anchors: fa = la, fb = lb after the pass
				cb.la[s] = add(cb.la[s], cb.fa[s]);
				cb.lb[s] = add(cb.lb[s], cb.fb[s]);
				cb.fa[s] = vzero<T>();
				cb.fb[s] = vzero<T>();
			}
		}
		if (!rec.gate)
		{
			continue;
		}
		Contact<T> c = loadContact<T>(tc[pos]);
		V<T> d0 = vzero<T>(), d1 = vzero<T>();
		Q<T> e0 = qzero<T>(), e1 = qzero<T>();
		V<T>& pAb = bc[c.a].dynamic ? x.adj[c.a].x : d0;
		Q<T>& qAb = bc[c.a].dynamic ? x.adj[c.a].q : e0;
		V<T>& pBb = bc[c.b].dynamic ? x.adj[c.b].x : d1;
		Q<T>& qBb = bc[c.b].dynamic ? x.adj[c.b].q : e1;
		T muB = T(0), imAb = T(0), imBb = T(0);
		M<T> iwAb, iwBb;
		iwAb.cx = iwAb.cy = iwAb.cz = vzero<T>();
		iwBb = iwAb;
		friction_rev(c, bc[c.a].invMass, bc[c.b].invMass, x.iw[c.a], x.iw[c.b], x.lamN + 4 * pos, rec.pA, rec.qA, rec.pB,
					 rec.qB, rec.lam, pAb, qAb, pBb, qBb, x.lamNBar + 4 * pos, x.lamTBar + 4 * pos, muB, imAb, imBb, iwAb,
					 iwBb, cb);
		if (bc[c.a].dynamic)
		{
			x.imBar[c.a] += imAb;
			x.iwBar[c.a].cx = add(x.iwBar[c.a].cx, iwAb.cx);
			x.iwBar[c.a].cy = add(x.iwBar[c.a].cy, iwAb.cy);
			x.iwBar[c.a].cz = add(x.iwBar[c.a].cz, iwAb.cz);
		}
		if (bc[c.b].dynamic)
		{
			x.imBar[c.b] += imBb;
			x.iwBar[c.b].cx = add(x.iwBar[c.b].cx, iwBb.cx);
			x.iwBar[c.b].cy = add(x.iwBar[c.b].cy, iwBb.cy);
			x.iwBar[c.b].cz = add(x.iwBar[c.b].cz, iwBb.cz);
		}
		scatterMaterials(x, c, muB, T(0));
	}
	// normal iterations, reverse
	for (int it = x.iterations - 1; it >= 0; --it)
	{
		for (ContactRun u = contactRunBegin(x, r, true); u.more; contactRunNext(x, r, u))
		{
			if (!u.mine)
			{
				continue;
			}
			const int pos = u.pos;
			Contact<T> c = loadContact<T>(tc[pos]);
			if (c.pointCount == 0)
			{
				continue;
			}
			const PoseRec<T>& rec = x.normRec[(size_t)it * x.positions + pos];
			V<T> d0 = vzero<T>(), d1 = vzero<T>();
			Q<T> e0 = qzero<T>(), e1 = qzero<T>();
			V<T>& pAb = bc[c.a].dynamic ? x.adj[c.a].x : d0;
			Q<T>& qAb = bc[c.a].dynamic ? x.adj[c.a].q : e0;
			V<T>& pBb = bc[c.b].dynamic ? x.adj[c.b].x : d1;
			Q<T>& qBb = bc[c.b].dynamic ? x.adj[c.b].q : e1;
			T imAb = T(0), imBb = T(0);
			normals_rev(c, x.prep[pos], bc[c.a].invMass, bc[c.b].invMass, x.maxCorrection, rec.pA, rec.qA, rec.pB,
						rec.qB, pAb, qAb, pBb, qBb, x.lamNBar + 4 * pos, x.prepBar[pos], imAb, imBb, x.cbar[pos]);
			if (bc[c.a].dynamic)
			{
				x.imBar[c.a] += imAb;
			}
			if (bc[c.b].dynamic)
			{
				x.imBar[c.b] += imBb;
			}
		}
	}
	// contact preparation (poses at preparation = the integrated ones)
	for (ContactRun u = contactRunBegin(x, r, false); u.more; contactRunNext(x, r, u))
	{
		if (!u.mine)
		{
			continue;
		}
		const int pos = u.pos;
		Contact<T> c = loadContact<T>(tc[pos]);
		// the states at preparation are the integrated ones, rebuilt here
		Body<T> sA = x.cur[c.a], sB = x.cur[c.b];
		if (bc[c.a].dynamic)
		{
			M<T> iw;
			integrate(x.start[(size_t)sub * x.bodyCount + c.a], bc[c.a], x.h, x.g, sA, iw);
		}
		if (bc[c.b].dynamic)
		{
			M<T> iw;
			integrate(x.start[(size_t)sub * x.bodyCount + c.b], bc[c.b], x.h, x.g, sB, iw);
		}
		const Q<T> qA1 = sA.q, qB1 = sB.q;
		Q<T> qAb = qzero<T>(), qBb = qzero<T>();
		T imAb = T(0), imBb = T(0);
		M<T> iwAb, iwBb;
		iwAb.cx = iwAb.cy = iwAb.cz = vzero<T>();
		iwBb = iwAb;
		prepare_rev(c, qA1, qB1, x.iw[c.a], x.iw[c.b], x.prep[pos], x.prepBar[pos], qAb, qBb, imAb, imBb, iwAb, iwBb,
					x.cbar[pos]);
		if (bc[c.a].dynamic)
		{
			x.adj[c.a].q = qadd(x.adj[c.a].q, qAb);
			x.imBar[c.a] += imAb;
			x.iwBar[c.a].cx = add(x.iwBar[c.a].cx, iwAb.cx);
			x.iwBar[c.a].cy = add(x.iwBar[c.a].cy, iwAb.cy);
			x.iwBar[c.a].cz = add(x.iwBar[c.a].cz, iwAb.cz);
		}
		if (bc[c.b].dynamic)
		{
			x.adj[c.b].q = qadd(x.adj[c.b].q, qBb);
			x.imBar[c.b] += imBb;
			x.iwBar[c.b].cx = add(x.iwBar[c.b].cx, iwBb.cx);
			x.iwBar[c.b].cy = add(x.iwBar[c.b].cy, iwBb.cy);
			x.iwBar[c.b].cz = add(x.iwBar[c.b].cz, iwBb.cz);
		}
		if (tc[pos].gen & kTapeGenPrepare)
		{
			// regenerated at the integrated poses; the manifold before it is
			// the previous substep's, or for substep 0 the one the step began
			// with (not on the tape when the narrowphase regenerated it too)
			const TapeContact* old = sub > 0 ? &x.contacts[(size_t)(sub - 1) * x.contactsPerSubstep + pos]
											 : ((tc[pos].gen & kTapeGenNarrow) ? nullptr : previousRecord(x, pos));
			const T margin = T(kGenSpeculativeBase) + x.h * len(m3d_diff::sub(sA.v, sB.v));
			reverseGeneration(x, tc[pos], old, sA.x, sA.q, sB.x, sB.q, margin, x.cbar[pos]);
		}
	}
	// integration
	for (int k = x.lane; k < r.bodyCount; k += x.width)
	{
		int i = x.bodies[r.bodyStart + k];
		if (!bc[i].dynamic)
		{
			continue;
		}
		Body<T> s1b = x.adj[i];
		s1b.v = vzero<T>();
		s1b.w = vzero<T>();
		BodyConstBar<T> cb;
		cb.invMass = T(0);
		cb.il = T(0);
		Body<T> s0b = x.adj0[i];
		integrate_rev(x.start[(size_t)sub * x.bodyCount + i], bc[i], x.h, x.g, s1b, x.iwBar[i], s0b, cb);
		x.ilBar[i] += cb.il;
		x.adj[i] = s0b;
	}
	teamSync(x);
}

// The slice of the per-substep records for substep `sub`: world inverse
// inertias, poses before reconstruction, prepared contacts, impulses, pose
// and velocity records (the work arrays hold one slice per substep; the
// adjoint scratch is shared).
template <typename T>
M3D_DIFF_HD IslandCtx<T> substepView(const IslandCtx<T>& x, int sub)
{
	IslandCtx<T> y = x;
	const size_t b = (size_t)sub * (size_t)x.bodyCount, p = (size_t)sub * (size_t)x.positions;
	y.iw = x.iw + b;
	y.x2 = x.x2 + b;
	y.q2 = x.q2 + b;
	y.prep = x.prep + p;
	y.lamN = x.lamN + 4 * p;
	y.lamT = x.lamT + 4 * p;
	y.normRec = x.normRec + p * (size_t)x.iterations;
	y.fricRec = x.fricRec + p;
	y.velRec = x.velRec + p;
	return y;
}

// One island through one step, recording: the forward pass with each
// substep's records in its own slice.  cur goes from the step's start to its
// end.
template <typename T>
M3D_DIFF_HD void islandStepRecord(const IslandCtx<T>& x)
{
	const TapeIsland& r = *x.island;
	for (int sub = 0; sub < x.substeps; ++sub)
	{
		substepForward(substepView(x, sub), r, sub, true);
	}
}

// One island through one step, in reverse, from the records of
// islandStepRecord: the adjoints of its bodies' state at the step's end in
// adj; on return adj holds the adjoints at the step's start and cur the state
// at the step's start.
template <typename T>
M3D_DIFF_HD void islandStepReverse(const IslandCtx<T>& x)
{
	const TapeIsland& r = *x.island;
	for (int sub = x.substeps - 1; sub >= 0; --sub)
	{
		substepReverse(substepView(x, sub), r, sub);
	}
	// cur: back to the step's start
	for (int k = x.lane; k < r.bodyCount; k += x.width)
	{
		int i = x.bodies[r.bodyStart + k];
		if (x.bc[i].dynamic)
		{
			x.cur[i] = x.start[i];
		}
	}
	teamSync(x);
	// manifolds the step's narrowphase regenerated at the step-start poses
	// (margin from the step-start velocities, as the narrowphase takes it);
	// the generations add into the bodies' adjoints: walked by level
	for (ContactRun u = contactRunBegin(x, r, false); u.more; contactRunNext(x, r, u))
	{
		if (!u.mine)
		{
			continue;
		}
		const int pos = u.pos;
		const TapeContact& rec = x.contacts[pos];
		if ((rec.gen & kTapeGenNarrow) && !(rec.gen & kTapeGenPrepare))
		{
			const Body<T>& A = x.cur[rec.a];
			const Body<T>& B = x.cur[rec.b];
			const T margin = T(kGenSpeculativeBase) + x.dt * len(m3d_diff::sub(A.v, B.v));
			reverseGeneration(x, rec, previousRecord(x, pos), A.x, A.q, B.x, B.q, margin, x.cbar[pos],
							  x.genJ != nullptr ? x.genJ + (size_t)pos * (kGenJRows * kGenJCols) : nullptr);
		}
	}
}

// One island through one step, backward: the state of its bodies at the
// step's start is in cur; the adjoints of their state at the step's end in
// adj.  On return adj holds the adjoints at the step's start and cur is
// unchanged.
template <typename T>
M3D_DIFF_HD void islandStepBackward(const IslandCtx<T>& x)
{
	islandStepRecord(x);
	islandStepReverse(x);
}

// One island through one step, forward only (the replay).
template <typename T>
M3D_DIFF_HD void islandStepForward(const IslandCtx<T>& x)
{
	const TapeIsland& r = *x.island;
	for (int sub = 0; sub < x.substeps; ++sub)
	{
		substepForward(x, r, sub, false);
	}
}

} // namespace m3d_diff

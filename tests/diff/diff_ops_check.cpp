// Finite-difference checks of the reverse (adjoint) functions of
// melon3d_b200/csrc/m3d_diff.h, in double precision on the CPU.  For each
// operation: random inputs, a random linear functional L of its outputs, the
// gradient of L from the reverse function, and the same gradient by central
// differences (step 1e-6).  Returns the largest relative error over all
// inputs (|g_rev - g_fd| / max(|g_fd|, 1)).  Test infrastructure only.
#include "m3d_diff.h"

#include <math.h>
#include <stdint.h>
#include <vector>

using namespace m3d_diff;
using D = double;

namespace
{

struct Rng
{
	uint64_t s;
	double u()
	{
		s = s * 6364136223846793005ull + 1442695040888963407ull;
		return (double)(s >> 11) * (1.0 / 9007199254740992.0);
	}
	double r(double a, double b) { return a + (b - a) * u(); }
};

V<D> rv(Rng& g, double a) { return v3<D>(g.r(-a, a), g.r(-a, a), g.r(-a, a)); }
Q<D> rq(Rng& g)
{
	Q<D> q = q4<D>(g.r(-1, 1), g.r(-1, 1), g.r(-1, 1), g.r(-1, 1));
	double l = sqrt(qdot(q, q));
	return qscale(1.0 / l, q);
}
M<D> rm(Rng& g)
{
	// symmetric, positive
	M<D> m;
	m.cx = v3<D>(g.r(0.5, 2), 0, 0);
	m.cy = v3<D>(0, g.r(0.5, 2), 0);
	m.cz = v3<D>(0, 0, g.r(0.5, 2));
	double a = g.r(-0.2, 0.2), b = g.r(-0.2, 0.2), c = g.r(-0.2, 0.2);
	m.cx.y = m.cy.x = a;
	m.cx.z = m.cz.x = b;
	m.cy.z = m.cz.y = c;
	return m;
}

// packing helpers
void put(std::vector<D>& v, V<D> a) { v.push_back(a.x), v.push_back(a.y), v.push_back(a.z); }
void put(std::vector<D>& v, Q<D> a) { v.push_back(a.x), v.push_back(a.y), v.push_back(a.z), v.push_back(a.w); }
void put(std::vector<D>& v, const M<D>& m) { put(v, m.cx), put(v, m.cy), put(v, m.cz); }
V<D> getv(const std::vector<D>& v, size_t& i)
{
	V<D> a = v3<D>(v[i], v[i + 1], v[i + 2]);
	i += 3;
	return a;
}
Q<D> getq(const std::vector<D>& v, size_t& i)
{
	Q<D> a = q4<D>(v[i], v[i + 1], v[i + 2], v[i + 3]);
	i += 4;
	return a;
}
M<D> getm(const std::vector<D>& v, size_t& i)
{
	M<D> m;
	m.cx = getv(v, i);
	m.cy = getv(v, i);
	m.cz = getv(v, i);
	return m;
}
double lin(const std::vector<D>& w, const std::vector<D>& out)
{
	double s = 0;
	for (size_t k = 0; k < out.size(); ++k)
		s += w[k] * out[k];
	return s;
}

template <typename F>
double fdCompare(const std::vector<D>& x0, const std::vector<D>& grad, F f, const std::vector<bool>* skip = nullptr)
{
	double worst = 0;
	for (size_t k = 0; k < x0.size(); ++k)
	{
		if (skip && (*skip)[k])
			continue;
		std::vector<D> a = x0, b = x0;
		double h = 1e-6;
		a[k] += h;
		b[k] -= h;
		double g = (f(a) - f(b)) / (2 * h);
		double e = fabs(grad[k] - g) / fmax(fabs(g), 1.0);
		worst = fmax(worst, e);
	}
	return worst;
}

Contact<D> randomContact(Rng& g, int pc, int shapeA, int shapeB, int curved)
{
	Contact<D> c;
	c.a = 0;
	c.b = 1;
	c.pointCount = pc;
	c.curved = curved;
	c.shapeA = shapeA;
	c.shapeB = shapeB;
	c.radiusA = g.r(0.1, 0.3);
	c.radiusB = g.r(0.1, 0.3);
	V<D> n = rv(g, 1);
	c.n = scale(1.0 / len(n), n);
	c.mu = g.r(0.2, 0.9);
	c.e = g.r(0.05, 0.3);
	c.rolling = g.r(0.01, 0.05);
	for (int s = 0; s < 4; ++s)
	{
		c.la[s] = rv(g, 0.3);
		c.lb[s] = rv(g, 0.3);
		c.off[s] = g.r(-0.05, -0.01);
		c.fa[s] = rv(g, 0.3);
		c.fb[s] = rv(g, 0.3);
		c.slip[s] = rv(g, 1);
	}
	return c;
}


// contact manifold data as a flat vector: n, la[4], lb[4], off[4], fa[4], fb[4]
void putContactData(std::vector<D>& v, const Contact<D>& c)
{
	put(v, c.n);
	for (int s = 0; s < 4; ++s)
		put(v, c.la[s]);
	for (int s = 0; s < 4; ++s)
		put(v, c.lb[s]);
	for (int s = 0; s < 4; ++s)
		v.push_back(c.off[s]);
	for (int s = 0; s < 4; ++s)
		put(v, c.fa[s]);
	for (int s = 0; s < 4; ++s)
		put(v, c.fb[s]);
}
void getContactData(const std::vector<D>& v, size_t& i, Contact<D>& c)
{
	c.n = getv(v, i);
	for (int s = 0; s < 4; ++s)
		c.la[s] = getv(v, i);
	for (int s = 0; s < 4; ++s)
		c.lb[s] = getv(v, i);
	for (int s = 0; s < 4; ++s)
		c.off[s] = v[i++];
	for (int s = 0; s < 4; ++s)
		c.fa[s] = getv(v, i);
	for (int s = 0; s < 4; ++s)
		c.fb[s] = getv(v, i);
}
void putBar(std::vector<D>& v, const ContactBar<D>& b)
{
	put(v, b.n);
	for (int s = 0; s < 4; ++s)
		put(v, b.la[s]);
	for (int s = 0; s < 4; ++s)
		put(v, b.lb[s]);
	for (int s = 0; s < 4; ++s)
		v.push_back(b.off[s]);
	for (int s = 0; s < 4; ++s)
		put(v, b.fa[s]);
	for (int s = 0; s < 4; ++s)
		put(v, b.fb[s]);
}

// poses of a touching pair: kind 0 box-box face (stacked, tilted), 1 box-box
// edge (crossed, rotated 45 deg), 2 sphere-box, 3 box-sphere (flipped order),
// 4 sphere-sphere
void pairFor(int kind, Rng& g, GenShape<D>& a, GenShape<D>& b, V<D>& xA, Q<D>& qA, V<D>& xB, Q<D>& qB)
{
	auto smallRot = [&](double ang) {
		V<D> ax = rv(g, 1);
		ax = scale(1.0 / len(ax), ax);
		double t = g.r(-ang, ang);
		return q4<D>(sin(t) * ax.x, sin(t) * ax.y, sin(t) * ax.z, cos(t));
	};
	a.type = b.type = kShapeBox;
	a.radius = b.radius = 0;
	a.he = v3<D>(g.r(0.2, 0.4), g.r(0.2, 0.4), g.r(0.2, 0.4));
	b.he = v3<D>(g.r(0.2, 0.4), g.r(0.2, 0.4), g.r(0.2, 0.4));
	xA = rv(g, 0.1);
	qA = smallRot(0.05);
	qB = smallRot(0.05);
	if (kind == 0)
	{
		xB = add(xA, v3<D>(g.r(-0.05, 0.05), a.he.y + b.he.y - 0.005, g.r(-0.05, 0.05)));
	}
	else if (kind == 1)
	{
		a.he = b.he = v3<D>(0.3, 0.3, 0.3);
		Q<D> ra = q4<D>(sin(M_PI / 8), 0, 0, cos(M_PI / 8)); // 45 deg about x
		Q<D> rb = q4<D>(0, 0, sin(M_PI / 8), cos(M_PI / 8)); // 45 deg about z
		qA = qmul(smallRot(0.02), ra);
		qB = qmul(smallRot(0.02), rb);
		xB = add(xA, v3<D>(g.r(-0.02, 0.02), 2 * 0.3 * sqrt(2.0) - 0.01, g.r(-0.02, 0.02)));
	}
	else if (kind == 2 || kind == 3)
	{
		GenShape<D> sph;
		sph.type = kShapeSphere;
		sph.radius = g.r(0.1, 0.3);
		sph.he = vzero<D>();
		GenShape<D> box = b;
		V<D> xs = add(xA, v3<D>(g.r(-0.1, 0.1), box.he.y + sph.radius - 0.005, g.r(-0.1, 0.1)));
		if (kind == 2)
		{
			a = sph, b = box;
			xB = xA;
			xA = xs;
		}
		else
		{
			a = box, b = sph;
			xB = xs;
		}
	}
	else
	{
		a.type = b.type = kShapeSphere;
		a.radius = g.r(0.1, 0.3);
		b.radius = g.r(0.1, 0.3);
		V<D> dir = rv(g, 1);
		dir = scale(1.0 / len(dir), dir);
		xB = madd(xA, a.radius + b.radius - 0.004, dir);
	}
}
} // namespace

extern "C"
{

double check_integrate(uint64_t seed)
{
	Rng g{ seed };
	BodyConst<D> c;
	c.invMass = g.r(0.5, 2);
	c.il = g.r(0.5, 3);
	c.gravityScale = 1;
	c.linearDamping = g.r(0, 0.1);
	c.angularDamping = g.r(0, 0.1);
	c.dynamic = 1;
	D h = 1.0 / 240.0;
	V<D> grav = v3<D>(0, -9.81, 0);
	std::vector<D> x;
	put(x, rv(g, 2));
	put(x, rq(g));
	put(x, rv(g, 2));
	// both rotation branches, and no spin at all (its adjoint is the
	// small-angle branch's limit)
	put(x, seed % 3 == 2 ? v3<D>(0, 0, 0) : rv(g, seed % 2 ? 20.0 : 0.5));
	x.push_back(c.il);
	std::vector<D> w(13 + 9);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto f = [&](const std::vector<D>& in) {
		size_t i = 0;
		Body<D> s0;
		s0.x = getv(in, i);
		s0.q = getq(in, i);
		s0.v = getv(in, i);
		s0.w = getv(in, i);
		BodyConst<D> cc = c;
		cc.il = in[i];
		Body<D> s1;
		M<D> iw;
		integrate(s0, cc, h, grav, s1, iw);
		std::vector<D> out;
		put(out, s1.x), put(out, s1.q), put(out, s1.v), put(out, s1.w), put(out, iw);
		return lin(w, out);
	};
	size_t i = 0;
	Body<D> s0;
	s0.x = getv(x, i);
	s0.q = getq(x, i);
	s0.v = getv(x, i);
	s0.w = getv(x, i);
	Body<D> s1b;
	size_t k = 0;
	s1b.x = getv(w, k);
	s1b.q = getq(w, k);
	s1b.v = getv(w, k);
	s1b.w = getv(w, k);
	M<D> iwb = getm(w, k);
	Body<D> s0b = bodyZero<D>();
	BodyConstBar<D> cb = { 0, 0 };
	integrate_rev(s0, c, h, grav, s1b, iwb, s0b, cb);
	std::vector<D> grad;
	put(grad, s0b.x), put(grad, s0b.q), put(grad, s0b.v), put(grad, s0b.w);
	grad.push_back(cb.il);
	// the inverse-inertia derivative is taken as isotropic (trace): exact for
	// il only when the rotation is orthonormal, which it is to rounding;
	// the rotation's effect on R d R^T is zero for isotropic d and is not
	// propagated, so compare with the iw part of L left out for q
	auto f2 = [&](const std::vector<D>& in) {
		size_t j = 0;
		Body<D> a;
		a.x = getv(in, j);
		a.q = getq(in, j);
		a.v = getv(in, j);
		a.w = getv(in, j);
		BodyConst<D> cc = c;
		cc.il = in[j];
		Body<D> s1;
		M<D> iw;
		integrate(a, cc, h, grav, s1, iw);
		// iw's rotation dependence removed: d * R R^T with R from the input
		// rotation renormalised exactly
		M<D> iso;
		iso.cx = v3<D>(cc.il, 0, 0);
		iso.cy = v3<D>(0, cc.il, 0);
		iso.cz = v3<D>(0, 0, cc.il);
		std::vector<D> out;
		put(out, s1.x), put(out, s1.q), put(out, s1.v), put(out, s1.w), put(out, iso);
		return lin(w, out);
	};
	(void)f;
	return fdCompare(x, grad, f2);
}

double check_prepare(uint64_t seed)
{
	Rng g{ seed };
	Contact<D> c = randomContact(g, 4, kShapeBox, (seed % 2) ? kShapeBox : kShapeSphere, 0);
	std::vector<D> x;
	put(x, rq(g));
	put(x, rq(g));
	x.push_back(g.r(0.5, 2));
	x.push_back(g.r(0.5, 2));
	put(x, rm(g));
	put(x, rm(g));
	std::vector<D> w(4 * 13);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto run = [&](const std::vector<D>& in, Prepared<D>& p) {
		size_t i = 0;
		Q<D> qA = getq(in, i), qB = getq(in, i);
		D imA = in[i++], imB = in[i++];
		M<D> iwA = getm(in, i), iwB = getm(in, i);
		preparedZero(p);
		prepare(c, qA, qB, imA, imB, iwA, iwB, p);
	};
	auto outv = [&](const Prepared<D>& p) {
		std::vector<D> out;
		for (int s = 0; s < 4; ++s)
		{
			put(out, p.rA[s]), put(out, p.rB[s]), put(out, p.jA[s]), put(out, p.jB[s]);
			out.push_back(p.wN[s]);
		}
		return out;
	};
	auto f = [&](const std::vector<D>& in) {
		Prepared<D> p;
		run(in, p);
		return lin(w, outv(p));
	};
	Prepared<D> p, pb;
	run(x, p);
	size_t k = 0;
	for (int s = 0; s < 4; ++s)
	{
		pb.rA[s] = getv(w, k), pb.rB[s] = getv(w, k), pb.jA[s] = getv(w, k), pb.jB[s] = getv(w, k);
		pb.wN[s] = w[k++];
	}
	size_t i = 0;
	Q<D> qA = getq(x, i), qB = getq(x, i);
	i += 2;
	M<D> iwA = getm(x, i), iwB = getm(x, i);
	Q<D> qAb = qzero<D>(), qBb = qzero<D>();
	D imAb = 0, imBb = 0;
	M<D> iwAb, iwBb;
	iwAb.cx = iwAb.cy = iwAb.cz = vzero<D>();
	iwBb = iwAb;
	ContactBar<D> cbar;
	contactBarZero(cbar);
	prepare_rev(c, qA, qB, iwA, iwB, p, pb, qAb, qBb, imAb, imBb, iwAb, iwBb, cbar);
	std::vector<D> grad;
	put(grad, qAb), put(grad, qBb);
	grad.push_back(imAb), grad.push_back(imBb);
	put(grad, iwAb), put(grad, iwBb);
	return fdCompare(x, grad, f);
}

// poses chosen so every point penetrates (sep < 0, above the cap)
double check_normals(uint64_t seed)
{
	Rng g{ seed };
	Contact<D> c = randomContact(g, 1 + (int)(seed % 4), kShapeBox, kShapeBox, 0);
	Prepared<D> p;
	preparedZero(p);
	for (int s = 0; s < 4; ++s)
	{
		p.jA[s] = rv(g, 0.5);
		p.jB[s] = rv(g, 0.5);
		p.wN[s] = g.r(1, 3);
	}
	V<D> pA = rv(g, 0.01), pB = rv(g, 0.01);
	Q<D> qA = rq(g), qB = rq(g);
	D imA = g.r(0.5, 2), imB = (seed % 3 == 0) ? 0.0 : g.r(0.5, 2);
	D maxC = 3.0 / 240.0;
	// offsets so that sep is clearly negative and above -maxC
	for (int s = 0; s < c.pointCount; ++s)
	{
		V<D> rA = rotate(qA, c.la[s]), rB = rotate(qB, c.lb[s]);
		D base = dot(sub(add(pB, rB), add(pA, rA)), c.n);
		c.off[s] = -base - g.r(0.002, 0.006);
	}
	std::vector<D> x;
	put(x, pA), put(x, qA), put(x, pB), put(x, qB);
	for (int s = 0; s < 4; ++s)
		x.push_back(g.r(0, 1)); // lambda in
	for (int s = 0; s < 4; ++s)
		put(x, p.jA[s]), put(x, p.jB[s]), x.push_back(p.wN[s]);
	x.push_back(imA), x.push_back(imB);
	std::vector<D> w(14 + 4);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto unpack = [&](const std::vector<D>& in, V<D>& a, Q<D>& qa, V<D>& b, Q<D>& qb, D* lam, Prepared<D>& pp, D& ia,
					  D& ib) {
		size_t i = 0;
		a = getv(in, i), qa = getq(in, i), b = getv(in, i), qb = getq(in, i);
		for (int s = 0; s < 4; ++s)
			lam[s] = in[i++];
		pp = p;
		for (int s = 0; s < 4; ++s)
			pp.jA[s] = getv(in, i), pp.jB[s] = getv(in, i), pp.wN[s] = in[i++];
		ia = in[i++], ib = in[i++];
	};
	auto f = [&](const std::vector<D>& in) {
		V<D> a, b;
		Q<D> qa, qb;
		D lam[4], ia, ib;
		Prepared<D> pp;
		unpack(in, a, qa, b, qb, lam, pp, ia, ib);
		normals(c, pp, ia, ib, maxC, a, qa, b, qb, lam);
		std::vector<D> out;
		put(out, a), put(out, qa), put(out, b), put(out, qb);
		for (int s = 0; s < 4; ++s)
			out.push_back(lam[s]);
		return lin(w, out);
	};
	V<D> a, b;
	Q<D> qa, qb;
	D lam[4], ia, ib;
	Prepared<D> pp;
	unpack(x, a, qa, b, qb, lam, pp, ia, ib);
	size_t k = 0;
	V<D> pAb = getv(w, k);
	Q<D> qAb = getq(w, k);
	V<D> pBb = getv(w, k);
	Q<D> qBb = getq(w, k);
	D lamb[4];
	for (int s = 0; s < 4; ++s)
		lamb[s] = w[k++];
	Prepared<D> pb;
	preparedZero(pb);
	D imAb = 0, imBb = 0;
	ContactBar<D> cbar;
	contactBarZero(cbar);
	normals_rev(c, pp, ia, ib, maxC, a, qa, b, qb, pAb, qAb, pBb, qBb, lamb, pb, imAb, imBb, cbar);
	std::vector<D> grad;
	put(grad, pAb), put(grad, qAb), put(grad, pBb), put(grad, qBb);
	for (int s = 0; s < 4; ++s)
		grad.push_back(lamb[s]);
	for (int s = 0; s < 4; ++s)
		put(grad, pb.jA[s]), put(grad, pb.jB[s]), grad.push_back(pb.wN[s]);
	grad.push_back(imAb), grad.push_back(ib == 0.0 ? 0.0 : imBb);
	std::vector<bool> skip(x.size(), false);
	if (ib == 0.0)
		skip[x.size() - 1] = true; // a static body stays static
	return fdCompare(x, grad, f, &skip);
}

double check_friction(uint64_t seed)
{
	Rng g{ seed };
	Contact<D> c = randomContact(g, 1 + (int)(seed % 4), kShapeBox, kShapeBox, 0);
	V<D> pA = rv(g, 0.05), pB = rv(g, 0.05);
	Q<D> qA = rq(g), qB = rq(g);
	D imA = g.r(0.5, 2), imB = (seed % 3 == 0) ? 0.0 : g.r(0.5, 2);
	M<D> iwA = rm(g), iwB = imB == 0.0 ? M<D>{ vzero<D>(), vzero<D>(), vzero<D>() } : rm(g);
	D lamN[4], lamT[4];
	for (int s = 0; s < 4; ++s)
	{
		// small budgets make some points take `allowed`, large ones `needed`
		lamN[s] = (s + seed) % 2 ? g.r(0.0005, 0.002) : g.r(0.5, 1.0);
		lamT[s] = 0;
	}
	std::vector<D> x;
	put(x, pA), put(x, qA), put(x, pB), put(x, qB);
	for (int s = 0; s < 4; ++s)
		x.push_back(lamN[s]);
	for (int s = 0; s < 4; ++s)
		x.push_back(lamT[s]);
	x.push_back(c.mu), x.push_back(imA), x.push_back(imB);
	put(x, iwA), put(x, iwB);
	std::vector<D> w(14 + 4);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto f = [&](const std::vector<D>& in) {
		size_t i = 0;
		V<D> a = getv(in, i);
		Q<D> qa = getq(in, i);
		V<D> b = getv(in, i);
		Q<D> qb = getq(in, i);
		D ln[4], lt[4];
		for (int s = 0; s < 4; ++s)
			ln[s] = in[i++];
		for (int s = 0; s < 4; ++s)
			lt[s] = in[i++];
		Contact<D> cc = c;
		cc.mu = in[i++];
		D ia = in[i++], ib = in[i++];
		M<D> ma = getm(in, i), mb = getm(in, i);
		friction(cc, ia, ib, ma, mb, ln, a, qa, b, qb, lt);
		std::vector<D> out;
		put(out, a), put(out, qa), put(out, b), put(out, qb);
		for (int s = 0; s < 4; ++s)
			out.push_back(lt[s]);
		return lin(w, out);
	};
	size_t k = 0;
	V<D> pAb = getv(w, k);
	Q<D> qAb = getq(w, k);
	V<D> pBb = getv(w, k);
	Q<D> qBb = getq(w, k);
	D lTb[4], lNb[4] = { 0, 0, 0, 0 };
	for (int s = 0; s < 4; ++s)
		lTb[s] = w[k++];
	D muB = 0, imAb = 0, imBb = 0;
	M<D> iwAb, iwBb;
	iwAb.cx = iwAb.cy = iwAb.cz = vzero<D>();
	iwBb = iwAb;
	ContactBar<D> cbar;
	contactBarZero(cbar);
	friction_rev(c, imA, imB, iwA, iwB, lamN, pA, qA, pB, qB, lamT, pAb, qAb, pBb, qBb, lNb, lTb, muB, imAb, imBb, iwAb,
				 iwBb, cbar);
	std::vector<D> grad;
	put(grad, pAb), put(grad, qAb), put(grad, pBb), put(grad, qBb);
	for (int s = 0; s < 4; ++s)
		grad.push_back(lNb[s]);
	for (int s = 0; s < 4; ++s)
		grad.push_back(lTb[s]);
	grad.push_back(muB), grad.push_back(imAb), grad.push_back(imBb);
	put(grad, iwAb), put(grad, iwBb);
	std::vector<bool> skip(x.size(), false);
	if (imB == 0.0)
	{
		skip[x.size() - 19] = true; // imB
		for (int t = 0; t < 9; ++t)
			skip[x.size() - 9 + t] = true; // iwB of a static body
	}
	return fdCompare(x, grad, f, &skip);
}

double check_reconstruct(uint64_t seed)
{
	Rng g{ seed };
	D invH = 240.0;
	V<D> x0 = rv(g, 1);
	Q<D> q0 = rq(g);
	// small or large rotation between q0 and q (both branches)
	V<D> ax = rv(g, 1);
	D ang = (seed % 2) ? 0.2 : 0.01;
	D l = len(ax);
	Q<D> dq = q4<D>(sin(ang) * ax.x / l, sin(ang) * ax.y / l, sin(ang) * ax.z / l, cos(ang));
	Q<D> q = qmul(dq, q0);
	V<D> xx = add(x0, rv(g, 0.01));
	std::vector<D> x;
	put(x, xx), put(x, q), put(x, x0), put(x, q0);
	std::vector<D> w(6);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto f = [&](const std::vector<D>& in) {
		size_t i = 0;
		V<D> a = getv(in, i);
		Q<D> qa = getq(in, i);
		V<D> a0 = getv(in, i);
		Q<D> qa0 = getq(in, i);
		V<D> v, ww;
		reconstruct(a, qa, a0, qa0, invH, v, ww);
		std::vector<D> out;
		put(out, v), put(out, ww);
		return lin(w, out);
	};
	V<D> xb = vzero<D>(), x0b = vzero<D>();
	Q<D> qb = qzero<D>(), q0b = qzero<D>();
	reconstruct_rev(xx, q, x0, q0, invH, v3<D>(w[0], w[1], w[2]), v3<D>(w[3], w[4], w[5]), xb, qb, x0b, q0b);
	std::vector<D> grad;
	put(grad, xb), put(grad, qb), put(grad, x0b), put(grad, q0b);
	return fdCompare(x, grad, f) / 240.0; // relative to the 1/h scale of the outputs
}

double check_velocity(uint64_t seed)
{
	Rng g{ seed };
	int curved = (int)(seed % 2);
	Contact<D> c = randomContact(g, 1 + (int)(seed % 4), kShapeBox, curved ? kShapeSphere : kShapeBox, curved);
	Prepared<D> p;
	preparedZero(p);
	for (int s = 0; s < 4; ++s)
	{
		p.rA[s] = rv(g, 0.3);
		p.rB[s] = rv(g, 0.3);
		p.jA[s] = rv(g, 0.5);
		p.jB[s] = rv(g, 0.5);
		p.wN[s] = g.r(1, 3);
		c.slip[s] = (s + seed) % 2 ? rv(g, 1) : v3<D>(0, 0, 0);
	}
	VelocityIn<D> in;
	in.imA = g.r(0.5, 2);
	in.imB = (seed % 3 == 0) ? 0.0 : g.r(0.5, 2);
	in.iwA = rm(g);
	in.iwB = in.imB == 0.0 ? M<D>{ vzero<D>(), vzero<D>(), vzero<D>() } : rm(g);
	in.qA = rq(g);
	in.qB = rq(g);
	in.pva = rv(g, 2), in.pwa = rv(g, 2), in.pvb = rv(g, 2), in.pwb = rv(g, 2);
	in.h = 1.0 / 240.0;
	in.gravityLen = 9.81;
	D lamN[4];
	for (int s = 0; s < 4; ++s)
		lamN[s] = (s + seed) % 3 ? g.r(0.001, 0.01) : g.r(0.00001, 0.0001);
	V<D> va = rv(g, 1), wa = rv(g, 1), vb = rv(g, 1), wb = rv(g, 1);
	std::vector<D> x;
	put(x, va), put(x, wa), put(x, vb), put(x, wb);
	put(x, in.pva), put(x, in.pwa), put(x, in.pvb), put(x, in.pwb);
	put(x, in.qA), put(x, in.qB);
	for (int s = 0; s < 4; ++s)
		x.push_back(lamN[s]);
	for (int s = 0; s < 4; ++s)
		put(x, p.rA[s]), put(x, p.rB[s]), put(x, p.jA[s]), put(x, p.jB[s]), x.push_back(p.wN[s]);
	x.push_back(c.mu), x.push_back(c.e), x.push_back(in.imA), x.push_back(in.imB);
	put(x, in.iwA), put(x, in.iwB);
	std::vector<D> w(12);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto unpack = [&](const std::vector<D>& v, V<D>& a, V<D>& aw, V<D>& b, V<D>& bw, VelocityIn<D>& ii, D* ln,
					  Prepared<D>& pp, Contact<D>& cc) {
		size_t i = 0;
		a = getv(v, i), aw = getv(v, i), b = getv(v, i), bw = getv(v, i);
		ii = in;
		ii.pva = getv(v, i), ii.pwa = getv(v, i), ii.pvb = getv(v, i), ii.pwb = getv(v, i);
		ii.qA = getq(v, i), ii.qB = getq(v, i);
		for (int s = 0; s < 4; ++s)
			ln[s] = v[i++];
		pp = p;
		for (int s = 0; s < 4; ++s)
			pp.rA[s] = getv(v, i), pp.rB[s] = getv(v, i), pp.jA[s] = getv(v, i), pp.jB[s] = getv(v, i),
			pp.wN[s] = v[i++];
		cc = c;
		cc.mu = v[i++];
		cc.e = v[i++];
		ii.imA = v[i++];
		ii.imB = v[i++];
		ii.iwA = getm(v, i);
		ii.iwB = getm(v, i);
	};
	auto f = [&](const std::vector<D>& v) {
		V<D> a, aw, b, bw;
		VelocityIn<D> ii;
		D ln[4];
		Prepared<D> pp;
		Contact<D> cc;
		unpack(v, a, aw, b, bw, ii, ln, pp, cc);
		velocity(cc, pp, ii, ln, a, aw, b, bw);
		std::vector<D> out;
		put(out, a), put(out, aw), put(out, b), put(out, bw);
		return lin(w, out);
	};
	V<D> vab = v3<D>(w[0], w[1], w[2]), wab = v3<D>(w[3], w[4], w[5]), vbb = v3<D>(w[6], w[7], w[8]),
		 wbb = v3<D>(w[9], w[10], w[11]);
	if (in.imB == 0.0)
	{
		// a static body's velocities are not outputs
		vbb = wbb = vzero<D>();
		w[6] = w[7] = w[8] = w[9] = w[10] = w[11] = 0;
	}
	Prepared<D> pb;
	preparedZero(pb);
	D lNb[4] = { 0, 0, 0, 0 };
	VelocityBar<D> b;
	b.imA = b.imB = b.mu = b.e = 0;
	b.iwA.cx = b.iwA.cy = b.iwA.cz = vzero<D>();
	b.iwB = b.iwA;
	b.qA = b.qB = qzero<D>();
	b.pva = b.pwa = b.pvb = b.pwb = vzero<D>();
	ContactBar<D> cbar;
	contactBarZero(cbar);
	velocity_rev(c, p, in, lamN, va, wa, vb, wb, vab, wab, vbb, wbb, pb, lNb, b, cbar);
	std::vector<D> grad;
	put(grad, vab), put(grad, wab), put(grad, vbb), put(grad, wbb);
	put(grad, b.pva), put(grad, b.pwa), put(grad, b.pvb), put(grad, b.pwb);
	put(grad, b.qA), put(grad, b.qB);
	for (int s = 0; s < 4; ++s)
		grad.push_back(lNb[s]);
	for (int s = 0; s < 4; ++s)
		put(grad, pb.rA[s]), put(grad, pb.rB[s]), put(grad, pb.jA[s]), put(grad, pb.jB[s]), grad.push_back(pb.wN[s]);
	grad.push_back(b.mu), grad.push_back(b.e), grad.push_back(b.imA), grad.push_back(b.imB);
	put(grad, b.iwA), put(grad, b.iwB);
	std::vector<bool> skip(x.size(), false);
	if (in.imB == 0.0)
	{
		skip[x.size() - 19] = true;
		for (int t = 0; t < 9; ++t)
			skip[x.size() - 9 + t] = true;
	}
	return fdCompare(x, grad, f, &skip);
}


// ---- adjoints of the manifold data (normal, anchors, offsets) ----------------------

double check_prepare_contact(uint64_t seed)
{
	Rng g{ seed };
	int curved = (int)(seed % 2);
	Contact<D> c = randomContact(g, 1 + (int)(seed % 4), curved ? kShapeSphere : kShapeBox, kShapeBox, curved);
	Q<D> qA = rq(g), qB = rq(g);
	D imA = g.r(0.5, 2), imB = g.r(0.5, 2);
	M<D> iwA = rm(g), iwB = rm(g);
	std::vector<D> x;
	putContactData(x, c);
	std::vector<D> w(4 * 13);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto outv = [&](const Prepared<D>& p) {
		std::vector<D> out;
		for (int s = 0; s < 4; ++s)
		{
			put(out, p.rA[s]), put(out, p.rB[s]), put(out, p.jA[s]), put(out, p.jB[s]);
			out.push_back(p.wN[s]);
		}
		return out;
	};
	auto f = [&](const std::vector<D>& in) {
		Contact<D> cc = c;
		size_t i = 0;
		getContactData(in, i, cc);
		Prepared<D> p;
		preparedZero(p);
		prepare(cc, qA, qB, imA, imB, iwA, iwB, p);
		return lin(w, outv(p));
	};
	Prepared<D> p, pb;
	preparedZero(p);
	prepare(c, qA, qB, imA, imB, iwA, iwB, p);
	size_t k = 0;
	for (int s = 0; s < 4; ++s)
	{
		pb.rA[s] = getv(w, k), pb.rB[s] = getv(w, k), pb.jA[s] = getv(w, k), pb.jB[s] = getv(w, k);
		pb.wN[s] = w[k++];
	}
	Q<D> qAb = qzero<D>(), qBb = qzero<D>();
	D imAb = 0, imBb = 0;
	M<D> iwAb, iwBb;
	iwAb.cx = iwAb.cy = iwAb.cz = vzero<D>();
	iwBb = iwAb;
	ContactBar<D> cb;
	contactBarZero(cb);
	prepare_rev(c, qA, qB, iwA, iwB, p, pb, qAb, qBb, imAb, imBb, iwAb, iwBb, cb);
	std::vector<D> grad;
	putBar(grad, cb);
	return fdCompare(x, grad, f);
}

double check_normals_contact(uint64_t seed)
{
	Rng g{ seed };
	Contact<D> c = randomContact(g, 1 + (int)(seed % 4), kShapeBox, kShapeBox, 0);
	Prepared<D> p;
	preparedZero(p);
	for (int s = 0; s < 4; ++s)
	{
		p.jA[s] = rv(g, 0.5);
		p.jB[s] = rv(g, 0.5);
		p.wN[s] = g.r(1, 3);
	}
	V<D> pA = rv(g, 0.01), pB = rv(g, 0.01);
	Q<D> qA = rq(g), qB = rq(g);
	D imA = g.r(0.5, 2), imB = (seed % 3 == 0) ? 0.0 : g.r(0.5, 2);
	D maxC = 3.0 / 240.0;
	for (int s = 0; s < c.pointCount; ++s)
	{
		V<D> rA = rotate(qA, c.la[s]), rB = rotate(qB, c.lb[s]);
		D base = dot(sub(add(pB, rB), add(pA, rA)), c.n);
		c.off[s] = -base - g.r(0.002, 0.006);
	}
	std::vector<D> x;
	putContactData(x, c);
	std::vector<D> w(14 + 4);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto f = [&](const std::vector<D>& in) {
		Contact<D> cc = c;
		size_t i = 0;
		getContactData(in, i, cc);
		V<D> a = pA, b = pB;
		Q<D> qa = qA, qb = qB;
		D lam[4] = { 0, 0, 0, 0 };
		normals(cc, p, imA, imB, maxC, a, qa, b, qb, lam);
		std::vector<D> out;
		put(out, a), put(out, qa), put(out, b), put(out, qb);
		for (int s = 0; s < 4; ++s)
			out.push_back(lam[s]);
		return lin(w, out);
	};
	size_t k = 0;
	V<D> pAb = getv(w, k);
	Q<D> qAb = getq(w, k);
	V<D> pBb = getv(w, k);
	Q<D> qBb = getq(w, k);
	D lamb[4];
	for (int s = 0; s < 4; ++s)
		lamb[s] = w[k++];
	Prepared<D> pb;
	preparedZero(pb);
	D imAb = 0, imBb = 0;
	ContactBar<D> cb;
	contactBarZero(cb);
	normals_rev(c, p, imA, imB, maxC, pA, qA, pB, qB, pAb, qAb, pBb, qBb, lamb, pb, imAb, imBb, cb);
	std::vector<D> grad;
	putBar(grad, cb);
	return fdCompare(x, grad, f);
}

double check_friction_contact(uint64_t seed)
{
	Rng g{ seed };
	Contact<D> c = randomContact(g, 1 + (int)(seed % 4), kShapeBox, kShapeBox, 0);
	V<D> pA = rv(g, 0.05), pB = rv(g, 0.05);
	Q<D> qA = rq(g), qB = rq(g);
	D imA = g.r(0.5, 2), imB = (seed % 3 == 0) ? 0.0 : g.r(0.5, 2);
	M<D> iwA = rm(g), iwB = imB == 0.0 ? M<D>{ vzero<D>(), vzero<D>(), vzero<D>() } : rm(g);
	D lamN[4], lamT[4];
	for (int s = 0; s < 4; ++s)
	{
		lamN[s] = (s + seed) % 2 ? g.r(0.0005, 0.002) : g.r(0.5, 1.0);
		lamT[s] = 0;
	}
	std::vector<D> x;
	putContactData(x, c);
	std::vector<D> w(14 + 4);
	for (auto& v : w)
		v = g.r(-1, 1);
	auto f = [&](const std::vector<D>& in) {
		Contact<D> cc = c;
		size_t i = 0;
		getContactData(in, i, cc);
		V<D> a = pA, b = pB;
		Q<D> qa = qA, qb = qB;
		D lt[4] = { 0, 0, 0, 0 };
		friction(cc, imA, imB, iwA, iwB, lamN, a, qa, b, qb, lt);
		std::vector<D> out;
		put(out, a), put(out, qa), put(out, b), put(out, qb);
		for (int s = 0; s < 4; ++s)
			out.push_back(lt[s]);
		return lin(w, out);
	};
	size_t k = 0;
	V<D> pAb = getv(w, k);
	Q<D> qAb = getq(w, k);
	V<D> pBb = getv(w, k);
	Q<D> qBb = getq(w, k);
	D lTb[4], lNb[4] = { 0, 0, 0, 0 };
	for (int s = 0; s < 4; ++s)
		lTb[s] = w[k++];
	D muB = 0, imAb = 0, imBb = 0;
	M<D> iwAb, iwBb;
	iwAb.cx = iwAb.cy = iwAb.cz = vzero<D>();
	iwBb = iwAb;
	ContactBar<D> cb;
	contactBarZero(cb);
	friction_rev(c, imA, imB, iwA, iwB, lamN, pA, qA, pB, qB, lamT, pAb, qAb, pBb, qBb, lNb, lTb, muB, imAb, imBb, iwAb,
				 iwBb, cb);
	std::vector<D> grad;
	putBar(grad, cb);
	return fdCompare(x, grad, f);
}

double check_velocity_contact(uint64_t seed)
{
	Rng g{ seed };
	int curved = (int)(seed % 2);
	Contact<D> c = randomContact(g, 1 + (int)(seed % 4), curved ? kShapeSphere : kShapeBox, kShapeBox, curved);
	Prepared<D> p;
	preparedZero(p);
	for (int s = 0; s < 4; ++s)
	{
		p.rA[s] = rv(g, 0.3);
		p.rB[s] = rv(g, 0.3);
		p.jA[s] = rv(g, 0.5);
		p.jB[s] = rv(g, 0.5);
		p.wN[s] = g.r(1, 3);
		c.slip[s] = (s + seed) % 2 ? rv(g, 1) : v3<D>(0, 0, 0);
	}
	VelocityIn<D> in;
	in.imA = g.r(0.5, 2);
	in.imB = (seed % 3 == 0) ? 0.0 : g.r(0.5, 2);
	in.iwA = rm(g);
	in.iwB = in.imB == 0.0 ? M<D>{ vzero<D>(), vzero<D>(), vzero<D>() } : rm(g);
	in.qA = rq(g);
	in.qB = rq(g);
	in.pva = rv(g, 2), in.pwa = rv(g, 2), in.pvb = rv(g, 2), in.pwb = rv(g, 2);
	in.h = 1.0 / 240.0;
	in.gravityLen = 9.81;
	D lamN[4];
	for (int s = 0; s < 4; ++s)
		lamN[s] = (s + seed) % 3 ? g.r(0.001, 0.01) : g.r(0.00001, 0.0001);
	V<D> va = rv(g, 1), wa = rv(g, 1), vb = rv(g, 1), wb = rv(g, 1);
	std::vector<D> x;
	putContactData(x, c);
	std::vector<D> w(12);
	for (auto& v : w)
		v = g.r(-1, 1);
	if (in.imB == 0.0)
		w[6] = w[7] = w[8] = w[9] = w[10] = w[11] = 0;
	auto f = [&](const std::vector<D>& v) {
		Contact<D> cc = c;
		size_t i = 0;
		getContactData(v, i, cc);
		V<D> a = va, aw = wa, b = vb, bw = wb;
		velocity(cc, p, in, lamN, a, aw, b, bw);
		std::vector<D> out;
		put(out, a), put(out, aw), put(out, b), put(out, bw);
		return lin(w, out);
	};
	V<D> vab = v3<D>(w[0], w[1], w[2]), wab = v3<D>(w[3], w[4], w[5]), vbb = v3<D>(w[6], w[7], w[8]),
		 wbb = v3<D>(w[9], w[10], w[11]);
	Prepared<D> pb;
	preparedZero(pb);
	D lNb[4] = { 0, 0, 0, 0 };
	VelocityBar<D> b;
	b.imA = b.imB = b.mu = b.e = 0;
	b.iwA.cx = b.iwA.cy = b.iwA.cz = vzero<D>();
	b.iwB = b.iwA;
	b.qA = b.qB = qzero<D>();
	b.pva = b.pwa = b.pvb = b.pwb = vzero<D>();
	ContactBar<D> cb;
	contactBarZero(cb);
	velocity_rev(c, p, in, lamN, va, wa, vb, wb, vab, wab, vbb, wbb, pb, lNb, b, cb);
	std::vector<D> grad;
	putBar(grad, cb);
	return fdCompare(x, grad, f);
}

// ---- manifold generation: dual-number Jacobian against central differences -------

double check_generation(uint64_t seed)
{
	Rng g{ seed };
	const int kind = (int)(seed % 5);
	GenShape<D> a, b;
	V<D> xA, xB;
	Q<D> qA, qB;
	pairFor(kind, g, a, b, xA, qA, xB, qB);
	const D margin = 0.02;
	GenManifold<D> m0;
	genManifold(a, xA, qA, b, xB, qB, margin, m0);
	if (m0.count == 0)
	{
		return 1e9; // the configuration must touch
	}
	typedef Dual<D, 14> S;
	GenShape<S> sa, sb;
	sa.type = a.type, sa.radius = S(a.radius), sa.he = v3<S>(S(a.he.x), S(a.he.y), S(a.he.z));
	sb.type = b.type, sb.radius = S(b.radius), sb.he = v3<S>(S(b.he.x), S(b.he.y), S(b.he.z));
	D in[14] = { xA.x, xA.y, xA.z, qA.x, qA.y, qA.z, qA.w, xB.x, xB.y, xB.z, qB.x, qB.y, qB.z, qB.w };
	S d[14];
	for (int k = 0; k < 14; ++k)
	{
		d[k] = S(in[k]);
		d[k].d[k] = 1;
	}
	GenManifold<S> md;
	genManifold(sa, v3<S>(d[0], d[1], d[2]), q4<S>(d[3], d[4], d[5], d[6]), sb, v3<S>(d[7], d[8], d[9]),
				q4<S>(d[10], d[11], d[12], d[13]), S(margin), md);
	if (md.count != m0.count)
	{
		return 1e9;
	}
	// outputs: n, then per point la, lb, off
	auto outputs = [&](const D* v, std::vector<D>& out) {
		GenManifold<D> m;
		genManifold(a, v3<D>(v[0], v[1], v[2]), q4<D>(v[3], v[4], v[5], v[6]), b, v3<D>(v[7], v[8], v[9]),
					q4<D>(v[10], v[11], v[12], v[13]), margin, m);
		out.clear();
		if (m.count != m0.count)
		{
			return false;
		}
		put(out, m.n);
		for (int i = 0; i < m.count; ++i)
		{
			if (m.p[i].id != m0.p[i].id)
				return false;
			put(out, m.p[i].la), put(out, m.p[i].lb), out.push_back(m.p[i].off);
		}
		return true;
	};
	double worst = 0;
	for (int k = 0; k < 14; ++k)
	{
		D vp[14], vm[14];
		for (int j = 0; j < 14; ++j)
			vp[j] = vm[j] = in[j];
		const double h = 1e-7;
		vp[k] += h;
		vm[k] -= h;
		std::vector<D> op, om;
		if (!outputs(vp, op) || !outputs(vm, om))
			continue; // a branch flipped within +-h
		std::vector<D> jac;
		jac.push_back(md.n.x.d[k]), jac.push_back(md.n.y.d[k]), jac.push_back(md.n.z.d[k]);
		for (int i = 0; i < md.count; ++i)
		{
			jac.push_back(md.p[i].la.x.d[k]), jac.push_back(md.p[i].la.y.d[k]), jac.push_back(md.p[i].la.z.d[k]);
			jac.push_back(md.p[i].lb.x.d[k]), jac.push_back(md.p[i].lb.y.d[k]), jac.push_back(md.p[i].lb.z.d[k]);
			jac.push_back(md.p[i].off.d[k]);
		}
		for (size_t o = 0; o < jac.size(); ++o)
		{
			double fd = (op[o] - om[o]) / (2 * h);
			worst = fmax(worst, fabs(jac[o] - fd) / fmax(fabs(fd), 1.0));
		}
	}
	return worst;
}
} // extern "C"

// Seeded synthetic scenes of the benchmark configurations, driven through a
// table of Melon3D C-API function pointers.  The same compiled code builds
// and steps a world of ANY library that exports the C API: the GPU library,
// or the reference built from its sources (used by the test suite and by the
// CPU-baseline leg of bench.py).  No public dataset is involved; every scene
// is generated from a fixed seed.
//
//   0  pyramid: 20-box base shrinking by one per row (210 unit boxes) on a
//      static 100x1x100 m ground, mu 0.6, e 0
//   1  streaming mixed rain: N bodies in thirds (spheres r~U[0.2,0.5],
//      capsules r~U[0.15,0.35] hh~U[0.2,0.6], boxes he~U[0.2,0.5]^3) over a
//      100x60x100 m volume, uniform random orientations, v~N(0,2) per axis,
//      mu~U[0.3,0.8], e~U[0,0.3]; every step the `churn` lowest dynamic
//      bodies (ties by index) are destroyed and as many new ones spawned
//   2  settled pile: nx x ny x nz lattice of boxes he 0.5 spaced 1.02 m with
//      +-0.01 m positional and +-1 deg rotational jitter, mu 0.6
//   3  raft: 15x15 touching boxes plus 5 droppers (one island > 300 contacts)
//   4  one world of the batched-worlds config (its index is the seed): its
//      own 12x1x12 m ground box, floor(exp(U[ln16, ln512])) bodies drawn from
//      the rain distributions inside a 10x10x10 m volume above it, and 0-4
//      ball or hinge joints between random body pairs, anchored at the pair's
//      midpoint (a > 0 fixes the body count, b > 0 leaves the joints out)
//   5  one world of the differentiable batch: a static 16x0.5x10 m incline
//      box tilted by theta~U[10,35] deg about z carrying an 8x8 grid of
//      bodies (alternately cubes he~U[0.1,0.3] and spheres r~U[0.1,0.3]),
//      each 0.01-0.3 m above the slope, v~N(0,1) per axis, mu~U[0.2,0.9],
//      e~U[0,0.3]; the incline has mu 1, e 0.  Sleep is off (b > 0: on);
//      0 < a < 64 sets the body count.
//   6  jointed raft: the raft of scene 3 (one island of > 300 contacts, the
//      coloured path) with every joint type inside it - rigid and soft
//      distance joints, ball joints, weld joints, hinges with a limit, a
//      motor, or both - plus a hinged chain with a limited link swinging from
//      a static pivot onto the raft, a motor-driven wheel on a static axle,
//      a soft distance pendulum and spheres, capsules and boxes dropped on
//      the raft (seeded); its joints all meet the one raft island once the
//      chain lands
//   7  settled stacks: an a x b grid of c-box stacks (unit cubes, 1.5 m
//      apart, mu 0.6) resting on a static ground box; they fall asleep after
//      about a second and then stay asleep (the fixed cost of a sleeping
//      scene)
#include "melon3d.h"

#include <algorithm>
#include <chrono>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <vector>

extern "C"
{

struct M3dApi
{
	m3d_world_def (*world_def_default)(void);
	m3d_body_def (*body_def_default)(void);
	m3d_shape_def (*shape_def_default)(void);
	m3d_world* (*world_create)(const m3d_world_def*);
	void (*world_destroy)(m3d_world*);
	void (*world_step)(m3d_world*, float, int);
	m3d_body_id (*body_create)(m3d_world*, const m3d_body_def*, const m3d_shape_def*);
	void (*body_destroy)(m3d_world*, m3d_body_id);
	m3d_vec3 (*body_position)(m3d_world*, m3d_body_id);
	m3d_profile (*world_profile)(m3d_world*);
	// optional: batch pose readback of the GPU library (NULL elsewhere)
	void (*read_poses)(m3d_world*, float*, float*, int32_t);
	// joints (scene 4)
	m3d_joint_id (*joint_create_ball)(m3d_world*, const m3d_ball_joint_def*);
	m3d_joint_id (*joint_create_hinge)(m3d_world*, const m3d_hinge_joint_def*);
	m3d_hinge_joint_def (*hinge_joint_def_default)(void);
	// joints (scene 6)
	m3d_joint_id (*joint_create_distance)(m3d_world*, const m3d_distance_joint_def*);
	m3d_joint_id (*joint_create_weld)(m3d_world*, const m3d_weld_joint_def*);
	m3d_weld_joint_def (*weld_joint_def_default)(void);
};

} // extern "C"

namespace
{

struct Rng
{
	uint64_t s;
	uint64_t next()
	{
		uint64_t z = (s += 0x9E3779B97F4A7C15ull);
		z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
		z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
		return z ^ (z >> 31);
	}
	double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
	float range(double a, double b) { return (float)(a + (b - a) * uniform()); }
	double normal()
	{
		double u1 = uniform(), u2 = uniform();
		if (u1 < 1e-300)
		{
			u1 = 1e-300;
		}
		return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
	}
	// uniform random rotation (Shoemake)
	m3d_quat quat()
	{
		double u1 = uniform(), u2 = uniform(), u3 = uniform();
		double a = sqrt(1.0 - u1), b = sqrt(u1);
		m3d_quat q = { (float)(a * sin(6.283185307179586 * u2)), (float)(a * cos(6.283185307179586 * u2)),
					   (float)(b * sin(6.283185307179586 * u3)), (float)(b * cos(6.283185307179586 * u3)) };
		return q;
	}
};

struct Scene
{
	M3dApi api;
	m3d_world* world = nullptr;
	int kind = 0;
	int churn = 0;
	Rng rng{ 0 };
	std::vector<m3d_body_id> dynamic; // live dynamic bodies, creation order
	std::vector<m3d_vec3> positions;  // creation pose of each entry of `dynamic` (scene 4)
	std::vector<m3d_quat> orientations;
	std::vector<float> pos, rot;
	double lastHostMs = 0.0;
};

void addGround(Scene& s, m3d_vec3 center, m3d_vec3 he)
{
	m3d_body_def bd = s.api.body_def_default();
	bd.type = M3D_BODY_STATIC;
	bd.position = center;
	m3d_shape_def sd = s.api.shape_def_default();
	sd.type = M3D_SHAPE_BOX;
	sd.halfExtents = he;
	s.api.body_create(s.world, &bd, &sd);
}

m3d_body_id addBox(Scene& s, m3d_vec3 p, m3d_quat q, m3d_vec3 he, float mu)
{
	m3d_body_def bd = s.api.body_def_default();
	bd.type = M3D_BODY_DYNAMIC;
	bd.position = p;
	bd.orientation = q;
	m3d_shape_def sd = s.api.shape_def_default();
	sd.type = M3D_SHAPE_BOX;
	sd.halfExtents = he;
	sd.friction = mu;
	m3d_body_id id = s.api.body_create(s.world, &bd, &sd);
	s.dynamic.push_back(id);
	return id;
}

// a body from the rain distributions at a uniform position in [lo, hi]
m3d_body_id spawnShape(Scene& s, int kind, m3d_vec3 lo, m3d_vec3 hi)
{
	Rng& r = s.rng;
	m3d_body_def bd = s.api.body_def_default();
	bd.type = M3D_BODY_DYNAMIC;
	bd.position = m3d_v3(r.range(lo.x, hi.x), r.range(lo.y, hi.y), r.range(lo.z, hi.z));
	bd.orientation = r.quat();
	bd.linearVelocity = m3d_v3((float)(2.0 * r.normal()), (float)(2.0 * r.normal()), (float)(2.0 * r.normal()));
	m3d_shape_def sd = s.api.shape_def_default();
	if (kind == 0)
	{
		sd.type = M3D_SHAPE_SPHERE;
		sd.radius = r.range(0.2, 0.5);
	}
	else if (kind == 1)
	{
		sd.type = M3D_SHAPE_CAPSULE;
		sd.radius = r.range(0.15, 0.35);
		sd.halfHeight = r.range(0.2, 0.6);
	}
	else
	{
		sd.type = M3D_SHAPE_BOX;
		sd.halfExtents = m3d_v3(r.range(0.2, 0.5), r.range(0.2, 0.5), r.range(0.2, 0.5));
	}
	sd.friction = r.range(0.3, 0.8);
	sd.restitution = r.range(0.0, 0.3);
	m3d_body_id id = s.api.body_create(s.world, &bd, &sd);
	s.dynamic.push_back(id);
	s.positions.push_back(bd.position);
	s.orientations.push_back(bd.orientation);
	return id;
}

m3d_body_id spawnRain(Scene& s, int kind)
{
	return spawnShape(s, kind, m3d_v3(-50.0f, 1.0f, -50.0f), m3d_v3(50.0f, 61.0f, 50.0f));
}

// joints of scene 4: pairs of distinct bodies, anchored at their midpoint
void addBatchJoints(Scene& s, int count)
{
	size_t n = s.dynamic.size();
	if (n < 2 || s.api.joint_create_ball == nullptr || s.api.joint_create_hinge == nullptr)
	{
		return;
	}
	std::vector<float> pos(n * 3), rot(n * 4);
	for (int j = 0; j < count; ++j)
	{
		size_t ia = (size_t)(s.rng.next() % n), ib = (size_t)(s.rng.next() % (n - 1));
		ib = ib >= ia ? ib + 1 : ib;
		bool hinge = (s.rng.next() & 1) != 0;
		m3d_body_id a = s.dynamic[ia], b = s.dynamic[ib];
		m3d_vec3 pa = s.positions[ia], pb = s.positions[ib];
		m3d_quat qa = s.orientations[ia], qb = s.orientations[ib];
		m3d_vec3 mid = m3d_scale(0.5f, m3d_add(pa, pb));
		m3d_vec3 la = m3d_inv_rotate(qa, m3d_sub(mid, pa)), lb = m3d_inv_rotate(qb, m3d_sub(mid, pb));
		if (hinge)
		{
			m3d_hinge_joint_def d = s.api.hinge_joint_def_default();
			d.bodyA = a;
			d.bodyB = b;
			d.localAnchorA = la;
			d.localAnchorB = lb;
			d.localAxisA = m3d_inv_rotate(qa, m3d_v3(0.0f, 1.0f, 0.0f));
			d.localAxisB = m3d_inv_rotate(qb, m3d_v3(0.0f, 1.0f, 0.0f));
			s.api.joint_create_hinge(s.world, &d);
		}
		else
		{
			m3d_ball_joint_def d;
			memset(&d, 0, sizeof(d));
			d.bodyA = a;
			d.bodyB = b;
			d.localAnchorA = la;
			d.localAnchorB = lb;
			s.api.joint_create_ball(s.world, &d);
		}
	}
}

// destroy the `churn` lowest dynamic bodies (ties by index), spawn as many
void churnStep(Scene& s)
{
	size_t n = s.dynamic.size();
	if (s.churn <= 0 || n == 0)
	{
		return;
	}
	std::vector<float> ys(n);
	if (s.api.read_poses != nullptr)
	{
		int32_t cap = 0;
		for (const m3d_body_id& id : s.dynamic)
		{
			cap = id.index + 1 > cap ? id.index + 1 : cap;
		}
		s.pos.resize((size_t)cap * 3);
		s.api.read_poses(s.world, s.pos.data(), nullptr, cap);
		for (size_t k = 0; k < n; ++k)
		{
			ys[k] = s.pos[(size_t)s.dynamic[k].index * 3 + 1];
		}
	}
	else
	{
		for (size_t k = 0; k < n; ++k)
		{
			ys[k] = s.api.body_position(s.world, s.dynamic[k]).y;
		}
	}
	std::vector<uint32_t> order(n);
	for (size_t k = 0; k < n; ++k)
	{
		order[k] = (uint32_t)k;
	}
	size_t m = (size_t)s.churn < n ? (size_t)s.churn : n;
	std::partial_sort(order.begin(), order.begin() + m, order.end(), [&](uint32_t a, uint32_t b) {
		if (ys[a] != ys[b])
		{
			return ys[a] < ys[b];
		}
		return s.dynamic[a].index < s.dynamic[b].index;
	});
	std::vector<uint32_t> victims(order.begin(), order.begin() + m);
	std::sort(victims.begin(), victims.end(),
			  [&](uint32_t a, uint32_t b) { return s.dynamic[a].index < s.dynamic[b].index; });
	std::vector<char> dead(n, 0);
	for (uint32_t k : victims)
	{
		s.api.body_destroy(s.world, s.dynamic[k]);
		dead[k] = 1;
	}
	std::vector<m3d_body_id> keep;
	keep.reserve(n);
	for (size_t k = 0; k < n; ++k)
	{
		if (!dead[k])
		{
			keep.push_back(s.dynamic[k]);
		}
	}
	s.dynamic.swap(keep);
	for (size_t k = 0; k < m; ++k)
	{
		spawnRain(s, (int)(s.rng.next() % 3));
	}
}


m3d_body_id addStatic(Scene& s, m3d_vec3 p, m3d_vec3 he)
{
	m3d_body_def bd = s.api.body_def_default();
	bd.type = M3D_BODY_STATIC;
	bd.position = p;
	m3d_shape_def sd = s.api.shape_def_default();
	sd.type = M3D_SHAPE_BOX;
	sd.halfExtents = he;
	return s.api.body_create(s.world, &bd, &sd);
}

m3d_body_id addDynamic(Scene& s, m3d_vec3 p, m3d_shape_def sd)
{
	m3d_body_def bd = s.api.body_def_default();
	bd.type = M3D_BODY_DYNAMIC;
	bd.position = p;
	m3d_body_id id = s.api.body_create(s.world, &bd, &sd);
	s.dynamic.push_back(id);
	return id;
}

m3d_shape_def boxShape(Scene& s, m3d_vec3 he)
{
	m3d_shape_def sd = s.api.shape_def_default();
	sd.type = M3D_SHAPE_BOX;
	sd.halfExtents = he;
	return sd;
}

// scene 6 (see the file header)
void buildJointedRaft(Scene& s)
{
	Rng& r = s.rng;
	addGround(s, m3d_v3(0.0f, -1.0f, 0.0f), m3d_v3(50.0f, 1.0f, 50.0f));
	const int N = 15;
	m3d_body_id raft[N][N];
	for (int gx = 0; gx < N; ++gx)
	{
		for (int gz = 0; gz < N; ++gz)
		{
			raft[gx][gz] = addBox(s, m3d_v3(1.0f * (float)gx - 7.0f, 0.5f, 1.0f * (float)gz - 7.0f), m3d_quat_identity(),
								  m3d_v3(0.501f, 0.5f, 0.501f), 0.6f);
		}
	}
	// joints between raft neighbours (joined pairs stop colliding): anchors
	// on the shared face, so every joint starts satisfied
	for (int k = 0; k < 24; ++k)
	{
		int gx = (int)(r.next() % (N - 1)), gz = (int)(r.next() % N);
		m3d_body_id a = raft[gx][gz], b = raft[gx + 1][gz];
		m3d_vec3 la = m3d_v3(0.5f, 0.0f, 0.0f), lb = m3d_v3(-0.5f, 0.0f, 0.0f);
		switch (k % 6)
		{
		case 0:
		case 1:
		{
			m3d_distance_joint_def d;
			memset(&d, 0, sizeof(d));
			d.bodyA = a;
			d.bodyB = b;
			d.localAnchorA = la;
			d.localAnchorB = lb;
			d.length = k % 6 == 0 ? 0.0f : 0.05f;
			d.hertz = k % 6 == 0 ? 0.0f : 3.0f;
			d.dampingRatio = k % 6 == 0 ? 0.0f : 0.7f;
			s.api.joint_create_distance(s.world, &d);
			break;
		}
		case 2:
		{
			m3d_ball_joint_def d;
			memset(&d, 0, sizeof(d));
			d.bodyA = a;
			d.bodyB = b;
			d.localAnchorA = la;
			d.localAnchorB = lb;
			s.api.joint_create_ball(s.world, &d);
			break;
		}
		case 3:
		{
			m3d_weld_joint_def d = s.api.weld_joint_def_default();
			d.bodyA = a;
			d.bodyB = b;
			d.localAnchorA = la;
			d.localAnchorB = lb;
			s.api.joint_create_weld(s.world, &d);
			break;
		}
		default:
		{
			m3d_hinge_joint_def d = s.api.hinge_joint_def_default();
			d.bodyA = a;
			d.bodyB = b;
			d.localAnchorA = la;
			d.localAnchorB = lb;
			d.localAxisA = m3d_v3(0.0f, 0.0f, 1.0f);
			d.enableLimit = k % 6 == 4 || k % 12 == 5;
			d.lowerAngle = -0.1f;
			d.upperAngle = 0.15f;
			d.enableMotor = k % 6 == 5;
			d.motorSpeed = 1.5f;
			d.maxMotorTorque = 40.0f;
			s.api.joint_create_hinge(s.world, &d);
			break;
		}
		}
	}
	// hinged chain from a static pivot above the raft's edge; the third link
	// has a limit, the last one a motor
	m3d_body_id prev = addStatic(s, m3d_v3(-7.0f, 6.0f, 0.0f), m3d_v3(0.1f, 0.1f, 0.1f));
	for (int i = 0; i < 6; ++i)
	{
		m3d_body_id link = addDynamic(s, m3d_v3(-7.0f + 0.9f * (float)(i + 1), 6.0f, 0.0f),
									  boxShape(s, m3d_v3(0.4f, 0.15f, 0.15f)));
		m3d_hinge_joint_def d = s.api.hinge_joint_def_default();
		d.bodyA = prev;
		d.bodyB = link;
		d.localAnchorA = i == 0 ? m3d_v3(0.0f, 0.0f, 0.0f) : m3d_v3(0.45f, 0.0f, 0.0f);
		d.localAnchorB = m3d_v3(-0.45f, 0.0f, 0.0f);
		d.localAxisA = m3d_v3(0.0f, 0.0f, 1.0f);
		d.enableLimit = i == 2;
		d.lowerAngle = -0.3f;
		d.upperAngle = 0.3f;
		d.enableMotor = i == 5;
		d.motorSpeed = -2.0f;
		d.maxMotorTorque = 5.0f;
		s.api.joint_create_hinge(s.world, &d);
		prev = link;
	}
	// motor-driven wheel on a static axle, limited to +-1 rad
	{
		m3d_body_id axle = addStatic(s, m3d_v3(12.0f, 3.0f, 0.0f), m3d_v3(0.1f, 0.1f, 0.1f));
		m3d_shape_def ws = s.api.shape_def_default();
		ws.type = M3D_SHAPE_CAPSULE;
		ws.radius = 0.2f;
		ws.halfHeight = 0.8f;
		m3d_body_id wheel = addDynamic(s, m3d_v3(12.0f, 3.0f, 0.0f), ws);
		m3d_hinge_joint_def d = s.api.hinge_joint_def_default();
		d.bodyA = axle;
		d.bodyB = wheel;
		d.localAxisA = m3d_v3(0.0f, 0.0f, 1.0f);
		d.enableMotor = true;
		d.motorSpeed = 4.0f;
		d.maxMotorTorque = 60.0f;
		d.enableLimit = true;
		d.lowerAngle = -1.0f;
		d.upperAngle = 1.0f;
		s.api.joint_create_hinge(s.world, &d);
	}
	// soft distance pendulum from a static hook
	{
		m3d_body_id hook = addStatic(s, m3d_v3(-12.0f, 5.0f, 0.0f), m3d_v3(0.1f, 0.1f, 0.1f));
		m3d_shape_def bs = s.api.shape_def_default();
		bs.type = M3D_SHAPE_SPHERE;
		bs.radius = 0.3f;
		m3d_body_id bob = addDynamic(s, m3d_v3(-10.5f, 5.0f, 0.5f), bs);
		m3d_distance_joint_def d;
		memset(&d, 0, sizeof(d));
		d.bodyA = hook;
		d.bodyB = bob;
		d.hertz = 2.0f;
		d.dampingRatio = 0.3f;
		s.api.joint_create_distance(s.world, &d);
	}
	// droppers on the raft
	for (int i = 0; i < 24; ++i)
	{
		spawnShape(s, i % 3, m3d_v3(-6.0f, 2.0f, -6.0f), m3d_v3(6.0f, 6.0f, 6.0f));
	}
}

} // namespace

extern "C"
{

// kind / params: see the file header.  a,b,c = pyramid base | rain count,
// churn | pile nx,ny,nz.
void* scn_create(const M3dApi* api, int kind, uint64_t seed, int a, int b, int c, int workers)
{
	Scene* s = new Scene();
	s->api = *api;
	s->kind = kind;
	s->rng.s = seed;
	m3d_world_def wd = s->api.world_def_default();
	if (workers > 0)
	{
		wd.workerCount = workers; // the reference's thread pool; the GPU world ignores it
	}
	if (kind == 5)
	{
		wd.enableSleep = b > 0;
	}
	s->world = s->api.world_create(&wd);
	if (s->world == nullptr)
	{
		delete s;
		return nullptr;
	}
	if (kind == 0)
	{
		addGround(*s, m3d_v3(0.0f, -0.5f, 0.0f), m3d_v3(50.0f, 0.5f, 50.0f));
		int base = a > 0 ? a : 20;
		const float he = 0.5f;
		for (int row = 0; row < base; ++row)
		{
			int count = base - row;
			float y = he + 2.0f * he * (float)row;
			float x0 = -he * (float)(count - 1);
			for (int i = 0; i < count; ++i)
			{
				addBox(*s, m3d_v3(x0 + 2.0f * he * (float)i, y, 0.0f), m3d_quat_identity(), m3d_v3(he, he, he), 0.6f);
			}
		}
	}
	else if (kind == 1)
	{
		addGround(*s, m3d_v3(0.0f, -0.5f, 0.0f), m3d_v3(50.0f, 0.5f, 50.0f));
		int count = a > 0 ? a : 20000;
		s->churn = b;
		for (int i = 0; i < count; ++i)
		{
			spawnRain(*s, i % 3);
		}
	}
	else if (kind == 2)
	{
		addGround(*s, m3d_v3(0.0f, -0.5f, 0.0f), m3d_v3(50.0f, 0.5f, 50.0f));
		int nx = a > 0 ? a : 50, ny = b > 0 ? b : 100, nz = c > 0 ? c : 50;
		const float sp = 1.02f;
		for (int j = 0; j < ny; ++j)
		{
			for (int i = 0; i < nx; ++i)
			{
				for (int k = 0; k < nz; ++k)
				{
					Rng& r = s->rng;
					m3d_vec3 p = m3d_v3(((float)i - 0.5f * (float)(nx - 1)) * sp + r.range(-0.01, 0.01),
										0.52f + (float)j * sp + r.range(-0.01, 0.01),
										((float)k - 0.5f * (float)(nz - 1)) * sp + r.range(-0.01, 0.01));
					m3d_vec3 axis = m3d_normalize(m3d_v3((float)r.normal(), (float)r.normal(), (float)r.normal()));
					float ang = r.range(-1.0, 1.0) * (M3D_PI / 180.0f);
					float hs = (float)sin(0.5 * (double)ang), hc = (float)cos(0.5 * (double)ang);
					m3d_quat q = { hs * axis.x, hs * axis.y, hs * axis.z, hc };
					addBox(*s, p, q, m3d_v3(0.5f, 0.5f, 0.5f), 0.6f);
				}
			}
		}
	}
	else if (kind == 4)
	{
		addGround(*s, m3d_v3(0.0f, -0.5f, 0.0f), m3d_v3(6.0f, 0.5f, 6.0f));
		double u = s->rng.uniform();
		int count = a > 0 ? a : (int)floor(exp(log(16.0) + u * (log(512.0) - log(16.0))));
		for (int i = 0; i < count; ++i)
		{
			spawnShape(*s, i % 3, m3d_v3(-5.0f, 0.5f, -5.0f), m3d_v3(5.0f, 10.5f, 5.0f));
		}
		int joints = (int)(s->rng.next() % 5);
		addBatchJoints(*s, b > 0 ? 0 : joints); // b > 0: no joints
	}
	else if (kind == 5)
	{
		Rng& r = s->rng;
		const double theta = (10.0 + 25.0 * r.uniform()) * 3.141592653589793 / 180.0;
		const m3d_quat q = { 0.0f, 0.0f, (float)sin(0.5 * theta), (float)cos(0.5 * theta) };
		m3d_body_def gd = s->api.body_def_default();
		gd.type = M3D_BODY_STATIC;
		gd.orientation = q;
		m3d_shape_def gs = s->api.shape_def_default();
		gs.type = M3D_SHAPE_BOX;
		gs.halfExtents = m3d_v3(8.0f, 0.25f, 5.0f);
		gs.friction = 1.0f;
		gs.restitution = 0.0f;
		s->api.body_create(s->world, &gd, &gs);
		const int count = a > 0 && a < 64 ? a : 64;
		for (int i = 0; i < count; ++i)
		{
			const int gx = i % 8, gz = i / 8;
			m3d_shape_def sd = s->api.shape_def_default();
			float size = r.range(0.1, 0.3);
			if (i % 2 == 0)
			{
				sd.type = M3D_SHAPE_BOX;
				sd.halfExtents = m3d_v3(size, size, size);
			}
			else
			{
				sd.type = M3D_SHAPE_SPHERE;
				sd.radius = size;
			}
			sd.friction = r.range(0.2, 0.9);
			sd.restitution = r.range(0.0, 0.3);
			const float gap = r.range(0.01, 0.3);
			m3d_vec3 local = m3d_v3(-2.8f + 0.8f * (float)gx, 0.25f + size + gap, -2.8f + 0.8f * (float)gz);
			m3d_body_def bd = s->api.body_def_default();
			bd.type = M3D_BODY_DYNAMIC;
			bd.position = m3d_rotate(q, local);
			bd.orientation = q;
			bd.linearVelocity = m3d_v3((float)r.normal(), (float)r.normal(), (float)r.normal());
			m3d_body_id id = s->api.body_create(s->world, &bd, &sd);
			s->dynamic.push_back(id);
			s->positions.push_back(bd.position);
			s->orientations.push_back(bd.orientation);
		}
	}
	else if (kind == 3)
	{
		addGround(*s, m3d_v3(0.0f, -1.0f, 0.0f), m3d_v3(50.0f, 1.0f, 50.0f));
		for (int gx = 0; gx < 15; ++gx)
		{
			for (int gz = 0; gz < 15; ++gz)
			{
				addBox(*s, m3d_v3(1.0f * (float)gx - 7.0f, 0.5f, 1.0f * (float)gz - 7.0f), m3d_quat_identity(),
					   m3d_v3(0.501f, 0.5f, 0.501f), 0.6f);
			}
		}
		for (int i = 0; i < 5; ++i)
		{
			addBox(*s, m3d_v3(2.0f * (float)i - 4.0f, 3.0f + 0.7f * (float)i, 0.5f * (float)i - 1.0f),
				   m3d_quat_identity(), m3d_v3(0.45f, 0.45f, 0.45f), 0.6f);
		}
	}
	else if (kind == 6)
	{
		buildJointedRaft(*s);
	}
	else if (kind == 7)
	{
		int nx = a > 0 ? a : 40, nz = b > 0 ? b : 30, ny = c > 0 ? c : 2;
		const float sp = 1.5f;
		float hx = 0.5f * sp * (float)nx + 5.0f, hz = 0.5f * sp * (float)nz + 5.0f;
		addGround(*s, m3d_v3(0.0f, -0.5f, 0.0f), m3d_v3(hx, 0.5f, hz));
		for (int i = 0; i < nx; ++i)
		{
			for (int k = 0; k < nz; ++k)
			{
				for (int j = 0; j < ny; ++j)
				{
					addBox(*s, m3d_v3(((float)i - 0.5f * (float)(nx - 1)) * sp, 0.5f + (float)j, ((float)k - 0.5f * (float)(nz - 1)) * sp),
						   m3d_quat_identity(), m3d_v3(0.5f, 0.5f, 0.5f), 0.6f);
				}
			}
		}
	}
	return s;
}

m3d_world* scn_world(void* scene) { return ((Scene*)scene)->world; }

int32_t scn_dynamic_count(void* scene) { return (int32_t)((Scene*)scene)->dynamic.size(); }

// Run `steps` steps at 60 Hz (churn included for the streaming scene).
// Returns the body-substeps advanced (dynamic bodies x substeps per step,
// summed) and writes the host wall time of the whole loop to *wallMs.
int64_t scn_run(void* scene, int steps, int substeps, double* wallMs, float* stepMsOut)
{
	Scene& s = *(Scene*)scene;
	int64_t bodySubsteps = 0;
	auto t0 = std::chrono::steady_clock::now();
	for (int i = 0; i < steps; ++i)
	{
		auto a = std::chrono::steady_clock::now();
		churnStep(s);
		s.api.world_step(s.world, 1.0f / 60.0f, substeps);
		bodySubsteps += (int64_t)s.dynamic.size() * substeps;
		if (stepMsOut != nullptr)
		{
			stepMsOut[i] = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - a).count();
		}
	}
	if (wallMs != nullptr)
	{
		*wallMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
	}
	return bodySubsteps;
}

// the streaming scene's destroy/spawn of one step, without stepping
void scn_churn(void* scene) { churnStep(*(Scene*)scene); }

// one step without the churn
void scn_step_only(void* scene, int substeps)
{
	Scene& s = *(Scene*)scene;
	s.api.world_step(s.world, 1.0f / 60.0f, substeps);
}

// dynamic bodies of world `seed` of the batched-worlds scene (scene 4 with
// a = 0), without building it
int32_t scn_batch_world_bodies(uint64_t seed)
{
	Rng r{ seed };
	double u = r.uniform();
	return (int32_t)floor(exp(log(16.0) + u * (log(512.0) - log(16.0))));
}

// ids of the live dynamic bodies (creation order)
int32_t scn_dynamic_ids(void* scene, m3d_body_id* out, int32_t cap)
{
	Scene& s = *(Scene*)scene;
	int32_t n = (int32_t)s.dynamic.size() < cap ? (int32_t)s.dynamic.size() : cap;
	for (int32_t i = 0; i < n; ++i)
	{
		out[i] = s.dynamic[i];
	}
	return n;
}

void scn_destroy(void* scene)
{
	Scene* s = (Scene*)scene;
	if (s->world != nullptr)
	{
		s->api.world_destroy(s->world);
	}
	delete s;
}

} // extern "C"

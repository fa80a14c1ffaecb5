// Oracle introspection shim — TEST INFRASTRUCTURE ONLY.
//
// Linked into the reference library built from the reference's own sources
// (see oracle/Makefile).  It reads the reference's internal world state
// (src/m3d_internal.h:602-685) and copies it into the neutral records of
// include/melon3d_debug.h, so the test suite can compare the GPU world with
// the reference step field by field: contact array order and manifolds
// (src/m3d_internal.h:154-229), island partitions (world->islandBodies, filled
// at src/world.cpp:1938-1956) and the greedy colouring of the last coloured
// island (world->colorBuckets / overflowContacts, src/xpbd.cpp:1179-1235).
// Nothing here is part of the product; the product never links it.
#include "m3d_internal.h"
#include "melon3d_debug.h"

#include <string.h>

using namespace m3d;

static void copy3(float* d, m3d_vec3 v)
{
	d[0] = v.x;
	d[1] = v.y;
	d[2] = v.z;
}

extern "C"
{

int32_t m3d_dbg_body_capacity(m3d_world* world) { return (int32_t)world->bodies.size(); }

void m3d_dbg_bodies(m3d_world* world, m3d_dbg_body* out, int32_t capacity)
{
	int32_t n = (int32_t)world->bodies.size();
	for (int32_t i = 0; i < n && i < capacity; ++i)
	{
		const Body& b = world->bodies[i];
		m3d_dbg_body& o = out[i];
		memset(&o, 0, sizeof(o));
		copy3(o.position, b.position);
		o.rotation[0] = b.rotation.x;
		o.rotation[1] = b.rotation.y;
		o.rotation[2] = b.rotation.z;
		o.rotation[3] = b.rotation.w;
		copy3(o.linearVelocity, b.linearVelocity);
		copy3(o.angularVelocity, b.angularVelocity);
		copy3(o.prevPosition, b.prevPosition);
		o.prevRotation[0] = b.prevRotation.x;
		o.prevRotation[1] = b.prevRotation.y;
		o.prevRotation[2] = b.prevRotation.z;
		o.prevRotation[3] = b.prevRotation.w;
		copy3(o.invInertiaWorld + 0, b.invInertiaWorld.cx);
		copy3(o.invInertiaWorld + 3, b.invInertiaWorld.cy);
		copy3(o.invInertiaWorld + 6, b.invInertiaWorld.cz);
		o.sleepTime = b.sleepTime;
		o.smoothedEnergy = b.smoothedEnergy;
		if (i < (int32_t)world->expandedAABBs.size())
		{
			copy3(o.fatLower, world->expandedAABBs[i].lowerBound);
			copy3(o.fatUpper, world->expandedAABBs[i].upperBound);
		}
		o.hasFatAABB = i < (int32_t)world->hasFatAABB.size() ? world->hasFatAABB[i] : 0;
		o.isAwake = b.isAwake ? 1 : 0;
		o.inUse = b.inUse ? 1 : 0;
	}
}

int32_t m3d_dbg_contact_count(m3d_world* world) { return (int32_t)world->contacts.size(); }

void m3d_dbg_contacts(m3d_world* world, m3d_dbg_contact* out, int32_t capacity)
{
	int32_t n = (int32_t)world->contacts.size();
	for (int32_t i = 0; i < n && i < capacity; ++i)
	{
		const Contact& c = world->contacts[i];
		m3d_dbg_contact& o = out[i];
		memset(&o, 0, sizeof(o));
		o.bodyA = c.bodyA;
		o.bodyB = c.bodyB;
		o.pointCount = c.manifold.pointCount;
		o.touching = c.touching ? 1 : 0;
		o.isSensor = c.isSensor ? 1 : 0;
		o.tunnelGuard = c.tunnelGuard ? 1 : 0;
		o.hasCache = c.hasCache ? 1 : 0;
		copy3(o.normal, c.manifold.normal);
		o.friction = c.friction;
		o.restitution = c.restitution;
		o.rollingResistance = c.rollingResistance;
		for (int32_t p = 0; p < c.manifold.pointCount && p < 4; ++p)
		{
			const ManifoldPoint& mp = c.manifold.points[p];
			m3d_dbg_point& q = o.points[p];
			copy3(q.localAnchorA, mp.localAnchorA);
			copy3(q.localAnchorB, mp.localAnchorB);
			copy3(q.frictionAnchorA, mp.frictionAnchorA);
			copy3(q.frictionAnchorB, mp.frictionAnchorB);
			q.separation = mp.separation;
			q.id = mp.id;
			q.lambdaN = mp.lambdaN;
			q.lambdaT = mp.lambdaT;
			q.separationOffset = mp.separationOffset;
			copy3(q.slipDir, mp.slipDir);
		}
	}
}

void m3d_dbg_island_labels(m3d_world* world, int32_t* out, int32_t capacity)
{
	for (int32_t i = 0; i < capacity; ++i)
	{
		out[i] = -1;
	}
	for (int32_t k = 0; k < world->islandUsed; ++k)
	{
		const std::vector<int32_t>& bodies = world->islandBodies[k];
		if (bodies.empty())
		{
			continue;
		}
		int32_t label = bodies[0];
		for (int32_t b : bodies)
		{
			label = b < label ? b : label;
		}
		for (int32_t b : bodies)
		{
			if (b < capacity)
			{
				out[b] = label;
			}
		}
	}
}

void m3d_dbg_contact_colors(m3d_world* world, int32_t* out, int32_t capacity)
{
	for (int32_t i = 0; i < capacity; ++i)
	{
		out[i] = -1;
	}
	for (int32_t c = 0; c < (int32_t)world->colorBuckets.size(); ++c)
	{
		for (int32_t ci : world->colorBuckets[c])
		{
			if (ci < capacity)
			{
				out[ci] = c;
			}
		}
	}
	for (int32_t ci : world->overflowContacts)
	{
		if (ci < capacity)
		{
			out[ci] = kMaxGraphColors;
		}
	}
}

} // extern "C"

/*
 * melon3d_debug.h — plain-C snapshot records used to compare two Melon3D
 * worlds field by field (the GPU world in libmelon3d_gpu.so and, in the test
 * suite, the CPU reference).  Both libraries fill these records through
 * functions with the same names and signatures:
 *
 *   int32_t m3d_dbg_body_capacity(m3d_world*);
 *   void    m3d_dbg_bodies(m3d_world*, m3d_dbg_body* out, int32_t capacity);
 *   int32_t m3d_dbg_contact_count(m3d_world*);
 *   void    m3d_dbg_contacts(m3d_world*, m3d_dbg_contact* out, int32_t capacity);
 *   void    m3d_dbg_island_labels(m3d_world*, int32_t* out, int32_t capacity);
 *   void    m3d_dbg_contact_colors(m3d_world*, int32_t* out, int32_t capacity);
 *
 * Island labels are canonical: the smallest body index of the island a
 * dynamic body belonged to in the last step, -1 for everything else.
 * Contact colours are the graph colour (0..7) of each contact in a coloured
 * island during the last step, 8 for the serial overflow bucket and -1 for a
 * contact that was not coloured.
 * The records carry no pointers and no C++ types; they are for tests and
 * debugging, not for the stepping path.
 */
#ifndef MELON3D_DEBUG_H
#define MELON3D_DEBUG_H

#include <stdint.h>

typedef struct m3d_dbg_point
{
	float localAnchorA[3];
	float localAnchorB[3];
	float frictionAnchorA[3];
	float frictionAnchorB[3];
	float separation;
	uint32_t id;
	float lambdaN;
	float lambdaT;
	float separationOffset;
	float slipDir[3];
} m3d_dbg_point;

typedef struct m3d_dbg_contact
{
	int32_t bodyA;
	int32_t bodyB;
	int32_t pointCount;
	uint8_t touching;
	uint8_t isSensor;
	uint8_t tunnelGuard;
	uint8_t hasCache;
	float normal[3];
	float friction;
	float restitution;
	float rollingResistance;
	m3d_dbg_point points[4];
} m3d_dbg_contact;

typedef struct m3d_dbg_body
{
	float position[3];
	float rotation[4];
	float linearVelocity[3];
	float angularVelocity[3];
	float prevPosition[3];
	float prevRotation[4];
	float invInertiaWorld[9]; /* columns cx, cy, cz */
	float sleepTime;
	float smoothedEnergy;
	float fatLower[3];
	float fatUpper[3];
	uint8_t hasFatAABB;
	uint8_t isAwake;
	uint8_t inUse;
	uint8_t pad;
} m3d_dbg_body;

#endif /* MELON3D_DEBUG_H */

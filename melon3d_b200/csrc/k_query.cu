// World queries on the device state: ray cast (Amanatides-Woo walk over the
// sorted cell entries plus the coarse lists), sphere cast, AABB overlap.
// (reference src/world.cpp:1081-1416)
#include "m3d_dev.cuh"
#include "m3d_solve.cuh"

#include <float.h>

namespace m3g
{

__device__ __forceinline__ uint64_t qPackCell(int64_t x, int64_t y, int64_t z)
{
	const int64_t offset = 1 << 20;
	uint64_t ux = (uint64_t)(x + offset) & 0x1FFFFFull;
	uint64_t uy = (uint64_t)(y + offset) & 0x1FFFFFull;
	uint64_t uz = (uint64_t)(z + offset) & 0x1FFFFFull;
	return (ux << 42) | (uy << 21) | uz;
}

struct RayState
{
	RayQueryOut out;
	float maxFraction;
};

__device__ void rayTestBody(const BodySoA& B, int32_t bi, uint32_t* stamps, uint32_t stamp, uint32_t mask, V3 origin,
							V3 translation, RayState& st)
{
	if (stamps[bi] == stamp)
	{
		return;
	}
	stamps[bi] = stamp;
	if (!(B.state[bi] & kStInUse) || (B.cold[bi].categoryBits & mask) == 0)
	{
		return;
	}
	float fraction;
	V3 normal;
	if (rayCastShape(B.cold[bi].shape, bodyXf(B, bi), origin, translation, &fraction, &normal) &&
		fraction < st.maxFraction)
	{
		st.maxFraction = fraction;
		st.out.hit = 1;
		st.out.body = bi;
		st.out.fraction = fraction;
		V3 p = madd(origin, fraction, translation);
		st.out.point[0] = p.x;
		st.out.point[1] = p.y;
		st.out.point[2] = p.z;
		st.out.normal[0] = normal.x;
		st.out.normal[1] = normal.y;
		st.out.normal[2] = normal.z;
	}
}

__device__ int64_t qLowerBound(const uint64_t* keys, int64_t n, uint64_t k)
{
	int64_t lo = 0, hi = n;
	while (lo < hi)
	{
		int64_t mid = (lo + hi) >> 1;
		if (keys[mid] < k)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo;
}

// one thread: the walk is inherently sequential and queries are rare
__global__ void kRayCast(BodySoA B, const uint64_t* actKeys, const uint32_t* actVals, int64_t nAct,
						 const uint64_t* stabKeys, const uint32_t* stabVals, int64_t nStab, const int32_t* actOver,
						 int32_t nAO, const int32_t* stabOver, int32_t nSO, uint32_t* stamps, uint32_t stamp,
						 uint32_t mask, V3 origin, V3 translation, float cs, RayQueryOut* out)
{
	M3G_KERNEL_BEGIN();
	RayState st;
	st.out.body = -1;
	V3 end = add(origin, translation);
	st.out.point[0] = end.x;
	st.out.point[1] = end.y;
	st.out.point[2] = end.z;
	st.out.normal[0] = st.out.normal[1] = st.out.normal[2] = 0.0f;
	st.out.fraction = 2.0f;
	st.out.hit = 0;
	st.maxFraction = 1.0f;

	for (int32_t k = 0; k < nAO; ++k)
	{
		rayTestBody(B, actOver[k], stamps, stamp, mask, origin, translation, st);
	}
	for (int32_t k = 0; k < nSO; ++k)
	{
		rayTestBody(B, stabOver[k], stamps, stamp, mask, origin, translation, st);
	}
	if (nAct > 0 || nStab > 0)
	{
		float inv = 1.0f / cs;
		int64_t cell[3] = { (int64_t)floorf(origin.x * inv), (int64_t)floorf(origin.y * inv),
							(int64_t)floorf(origin.z * inv) };
		float d[3] = { translation.x, translation.y, translation.z };
		float o[3] = { origin.x, origin.y, origin.z };
		int64_t stepDir[3];
		float tMax[3], tDelta[3];
		for (int k = 0; k < 3; ++k)
		{
			if (fabsf(d[k]) < 1e-12f)
			{
				stepDir[k] = 0;
				tMax[k] = FLT_MAX;
				tDelta[k] = FLT_MAX;
			}
			else
			{
				stepDir[k] = d[k] > 0.0f ? 1 : -1;
				float boundary = (float)(cell[k] + (stepDir[k] > 0 ? 1 : 0)) * cs;
				tMax[k] = (boundary - o[k]) / d[k];
				tDelta[k] = cs / fabsf(d[k]);
			}
		}
		float t = 0.0f;
		for (int guard = 0; guard < 4096 && t <= st.maxFraction; ++guard)
		{
			V3 probe = v3(((float)cell[0] + 0.5f) * cs, ((float)cell[1] + 0.5f) * cs, ((float)cell[2] + 0.5f) * cs);
			uint64_t key = qPackCell((int64_t)floorf(probe.x * inv), (int64_t)floorf(probe.y * inv),
									 (int64_t)floorf(probe.z * inv));
			for (int64_t e = qLowerBound(actKeys, nAct, key); e < nAct && actKeys[e] == key; ++e)
			{
				rayTestBody(B, (int32_t)actVals[e], stamps, stamp, mask, origin, translation, st);
			}
			for (int64_t e = qLowerBound(stabKeys, nStab, key); e < nStab && stabKeys[e] == key; ++e)
			{
				rayTestBody(B, (int32_t)stabVals[e], stamps, stamp, mask, origin, translation, st);
			}
			int axis = 0;
			if (tMax[1] < tMax[axis])
				axis = 1;
			if (tMax[2] < tMax[axis])
				axis = 2;
			t = tMax[axis];
			if (t > 1.0f || stepDir[axis] == 0)
			{
				break;
			}
			cell[axis] += stepDir[axis];
			tMax[axis] += tDelta[axis];
		}
	}
	*out = st.out;
}

void launchRayCast(DevWorld& w, int32_t n, V3 origin, V3 translation, uint32_t maskBits, float cellSize,
				   RayQueryOut* hostOut)
{
	static uint32_t stampCounter = 0;
	w.colorMask.ensureZeroed((size_t)(w.bodyCap + 1) * sizeof(uint32_t), w.stream); // stamps share this buffer
	w.queryOut.ensure(sizeof(RayQueryOut) * 2);
	// stamps live in a buffer other kernels overwrite; restart from a cleared state
	cudaMemsetAsync(w.colorMask.ptr, 0, (size_t)(w.bodyCap + 1) * sizeof(uint32_t), w.stream);
	stampCounter = 1;
	(void)n;
	M3G_LAUNCH(kRayCast, 1, 1, w.stream, w.B, w.activeKeys.as<uint64_t>(), w.activeVals.as<uint32_t>(), w.activeEntries,
									 w.stableKeys.as<uint64_t>(), w.stableVals.as<uint32_t>(), w.stableEntries,
									 w.activeOver.as<int32_t>(), w.activeOverCount, w.stableOver.as<int32_t>(),
									 w.stableOverCount, w.colorMask.as<uint32_t>(), stampCounter, maskBits, origin,
									 translation, cellSize, w.queryOut.as<RayQueryOut>());
	cudaMemcpyAsync(hostOut, w.queryOut.ptr, sizeof(RayQueryOut), cudaMemcpyDeviceToHost, w.stream);
	cudaStreamSynchronize(w.stream);
}

// signed distance to the shape surface and the closest surface point
// (reference src/world.cpp:1218-1284)
__device__ float pointShapeClosest(const Shape& s, Xf xf, V3 p, V3* closestOut)
{
	switch (s.type)
	{
		case kSphere:
		{
			V3 d = sub(p, xf.p);
			float l = len(d);
			V3 dir = l > 1e-9f ? scale(1.0f / l, d) : v3(0.0f, 1.0f, 0.0f);
			*closestOut = madd(xf.p, s.radius, dir);
			return l - s.radius;
		}
		case kCapsule:
		{
			V3 axis = rotate(xf.q, v3(0.0f, 1.0f, 0.0f));
			V3 pa = madd(xf.p, -s.halfHeight, axis);
			V3 ab = scale(2.0f * s.halfHeight, axis);
			float denom = dot(ab, ab);
			float t = denom > 1e-12f ? dot(sub(p, pa), ab) / denom : 0.0f;
			t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
			V3 c = madd(pa, t, ab);
			V3 d = sub(p, c);
			float l = len(d);
			V3 dir = l > 1e-9f ? scale(1.0f / l, d) : v3(0.0f, 1.0f, 0.0f);
			*closestOut = madd(c, s.radius, dir);
			return l - s.radius;
		}
		default:
		{
			V3 lp = xfInvPoint(xf, p);
			V3 he = s.he;
			V3 cl = v3(lp.x < -he.x ? -he.x : (lp.x > he.x ? he.x : lp.x), lp.y < -he.y ? -he.y : (lp.y > he.y ? he.y : lp.y),
					   lp.z < -he.z ? -he.z : (lp.z > he.z ? he.z : lp.z));
			V3 diff = sub(lp, cl);
			float dist2 = len2(diff);
			if (dist2 > 0.0f)
			{
				*closestOut = xfPoint(xf, cl);
				return sqrtf(dist2);
			}
			float dx = he.x - fabsf(lp.x);
			float dy = he.y - fabsf(lp.y);
			float dz = he.z - fabsf(lp.z);
			V3 face = lp;
			float depth;
			if (dx <= dy && dx <= dz)
			{
				face.x = lp.x >= 0.0f ? he.x : -he.x;
				depth = dx;
			}
			else if (dy <= dz)
			{
				face.y = lp.y >= 0.0f ? he.y : -he.y;
				depth = dy;
			}
			else
			{
				face.z = lp.z >= 0.0f ? he.z : -he.z;
				depth = dz;
			}
			*closestOut = xfPoint(xf, face);
			return -depth;
		}
	}
}

// Each body's own sphere-cast candidate, independent of the others; the
// serial reference loop keeps the first start-overlap body, else the smallest
// fraction with the lowest index winning ties, which the two atomicMin keys
// reproduce.  (reference src/world.cpp:1286-1392)
struct CastRec
{
	float fraction;
	float point[3];
	float normal[3];
};

__global__ void kSphereCast(BodySoA B, int32_t n, V3 origin, float radius, V3 translation, uint32_t mask, CastRec* recs,
							unsigned long long* keys)
{
	M3G_KERNEL_BEGIN();
	int bi = blockIdx.x * blockDim.x + threadIdx.x;
	if (bi >= n)
	{
		return;
	}
	if (!(B.state[bi] & kStInUse) || (B.cold[bi].categoryBits & mask) == 0)
	{
		return;
	}
	V3 end = add(origin, translation);
	V3 pad = v3(radius + 1e-3f, radius + 1e-3f, radius + 1e-3f);
	Box sweep;
	sweep.lo = sub(vmin(origin, end), pad);
	sweep.hi = add(vmax(origin, end), pad);
	float l = len(translation);
	const Shape& shape = B.cold[bi].shape;
	Xf xf = bodyXf(B, bi);
	if (!overlap(sweep, shapeAABB(shape, xf)))
	{
		return;
	}
	CastRec rec;
	{
		V3 closest;
		float rawDist = pointShapeClosest(shape, xf, origin, &closest);
		if (rawDist - radius < 1e-4f)
		{
			rec.fraction = 0.0f;
			rec.point[0] = closest.x;
			rec.point[1] = closest.y;
			rec.point[2] = closest.z;
			V3 outward = rawDist >= 0.0f ? sub(origin, closest) : sub(closest, origin);
			V3 nn = normalize(outward);
			rec.normal[0] = nn.x;
			rec.normal[1] = nn.y;
			rec.normal[2] = nn.z;
			recs[bi] = rec;
			atomicMin(&keys[0], (unsigned long long)bi);
			return;
		}
	}
	if (shape.type == kSphere || shape.type == kCapsule)
	{
		Shape infl = shape;
		infl.radius += radius;
		float fraction;
		V3 normal;
		if (rayCastShape(infl, xf, origin, translation, &fraction, &normal))
		{
			V3 center = madd(origin, fraction, translation);
			V3 p = madd(center, -radius, normal);
			rec.fraction = fraction;
			rec.point[0] = p.x;
			rec.point[1] = p.y;
			rec.point[2] = p.z;
			rec.normal[0] = normal.x;
			rec.normal[1] = normal.y;
			rec.normal[2] = normal.z;
			recs[bi] = rec;
			atomicMin(&keys[1], ((unsigned long long)__float_as_uint(fraction) << 32) | (unsigned)bi);
		}
		return;
	}
	float t = 0.0f;
	for (int iter = 0; iter < 128; ++iter)
	{
		V3 p = madd(origin, t, translation);
		V3 closest;
		float rawDist = pointShapeClosest(shape, xf, p, &closest);
		float d = rawDist - radius;
		if (d < 1e-4f)
		{
			rec.fraction = t;
			rec.point[0] = closest.x;
			rec.point[1] = closest.y;
			rec.point[2] = closest.z;
			V3 outward = rawDist >= 0.0f ? sub(p, closest) : sub(closest, p);
			V3 nn = normalize(outward);
			rec.normal[0] = nn.x;
			rec.normal[1] = nn.y;
			rec.normal[2] = nn.z;
			recs[bi] = rec;
			atomicMin(&keys[1], ((unsigned long long)__float_as_uint(t) << 32) | (unsigned)bi);
			return;
		}
		if (l < 1e-9f)
		{
			return;
		}
		t += d / l;
		if (t > 1.0f)
		{
			return;
		}
	}
}

__global__ void kSphereCastPick(const CastRec* recs, const unsigned long long* keys, V3 origin, V3 translation,
								RayQueryOut* out)
{
	M3G_KERNEL_BEGIN();
	RayQueryOut r;
	V3 end = add(origin, translation);
	r.body = -1;
	r.point[0] = end.x;
	r.point[1] = end.y;
	r.point[2] = end.z;
	r.normal[0] = r.normal[1] = r.normal[2] = 0.0f;
	r.fraction = 2.0f;
	r.hit = 0;
	int32_t bi = -1;
	if (keys[0] != ~0ull)
	{
		bi = (int32_t)keys[0];
	}
	else if (keys[1] != ~0ull)
	{
		bi = (int32_t)(keys[1] & 0xFFFFFFFFull);
	}
	if (bi >= 0)
	{
		const CastRec& c = recs[bi];
		r.body = bi;
		r.hit = 1;
		r.fraction = c.fraction;
		for (int k = 0; k < 3; ++k)
		{
			r.point[k] = c.point[k];
			r.normal[k] = c.normal[k];
		}
	}
	*out = r;
}

void launchSphereCast(DevWorld& w, int32_t n, V3 origin, float radius, V3 translation, uint32_t maskBits,
					  RayQueryOut* hostOut)
{
	radius = radius > 0.0f ? radius : 0.0f;
	w.queryOut.ensure(sizeof(RayQueryOut) + 16 + sizeof(CastRec) * (size_t)(n + 1));
	char* base = (char*)w.queryOut.ptr;
	RayQueryOut* out = (RayQueryOut*)base;
	unsigned long long* keys = (unsigned long long*)(base + 64);
	CastRec* recs = (CastRec*)(base + 128);
	w.queryOut.ensure(128 + sizeof(CastRec) * (size_t)(n + 1));
	base = (char*)w.queryOut.ptr;
	out = (RayQueryOut*)base;
	keys = (unsigned long long*)(base + 64);
	recs = (CastRec*)(base + 128);
	cudaMemsetAsync(keys, 0xFF, 2 * sizeof(unsigned long long), w.stream);
	if (n > 0)
	{
		M3G_LAUNCH(kSphereCast, blocksFor(n, 128), 128, w.stream, w.B, n, origin, radius, translation, maskBits, recs, keys);
	}
	M3G_LAUNCH(kSphereCastPick, 1, 1, w.stream, recs, keys, origin, translation, out);
	cudaMemcpyAsync(hostOut, out, sizeof(RayQueryOut), cudaMemcpyDeviceToHost, w.stream);
	cudaStreamSynchronize(w.stream);
}

static_assert(sizeof(CastRec) == kCastRecBytes, "scratch sizing of the fixed-buffer sphere cast");

size_t sphereCastScratchBytes(int32_t n) { return 128 + sizeof(CastRec) * (size_t)(n + 1); }

// The same two kernels over a caller-provided scratch block laid out as
// above (result at 0, the two pick keys at 64, per-body records at 128).
// Only the keys need a defined start value; a record is read only for the
// body whose key won, which this call wrote.
void launchSphereCastInto(DevWorld& w, int32_t n, V3 origin, float radius, V3 translation, uint32_t maskBits,
						  void* scratch, RayQueryOut* hostOut)
{
	radius = radius > 0.0f ? radius : 0.0f;
	char* base = (char*)scratch;
	RayQueryOut* out = (RayQueryOut*)base;
	unsigned long long* keys = (unsigned long long*)(base + 64);
	CastRec* recs = (CastRec*)(base + 128);
	cudaMemsetAsync(keys, 0xFF, 2 * sizeof(unsigned long long), w.stream);
	if (n > 0)
	{
		M3G_LAUNCH(kSphereCast, blocksFor(n, 128), 128, w.stream, w.B, n, origin, radius, translation, maskBits, recs, keys);
	}
	M3G_LAUNCH(kSphereCastPick, 1, 1, w.stream, recs, keys, origin, translation, out);
	cudaMemcpyAsync(hostOut, out, sizeof(RayQueryOut), cudaMemcpyDeviceToHost, w.stream);
	cudaStreamSynchronize(w.stream);
}

__global__ void kOverlap(BodySoA B, int32_t n, Box box, uint8_t* flags)
{
	M3G_KERNEL_BEGIN();
	int bi = blockIdx.x * blockDim.x + threadIdx.x;
	if (bi >= n)
	{
		return;
	}
	uint8_t f = 0;
	if ((B.state[bi] & kStInUse) && overlap(box, shapeAABB(B.cold[bi].shape, bodyXf(B, bi))))
	{
		f = 1;
	}
	flags[bi] = f;
}

void launchOverlap(DevWorld& w, int32_t n, Box box, uint8_t* hostFlags)
{
	if (n <= 0)
	{
		return;
	}
	w.queryOut.ensure((size_t)n + 64);
	M3G_LAUNCH(kOverlap, blocksFor(n, 256), 256, w.stream, w.B, n, box, w.queryOut.as<uint8_t>());
	cudaMemcpyAsync(hostFlags, w.queryOut.ptr, (size_t)n, cudaMemcpyDeviceToHost, w.stream);
	cudaStreamSynchronize(w.stream);
}

} // namespace m3g

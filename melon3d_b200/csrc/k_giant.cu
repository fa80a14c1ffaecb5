// Graph-coloured solve of giant islands on the whole GPU.
//
// The reference solves an island of >= 300 contacts with a greedy first-fit
// colouring in contact order and colour-parallel projection
// (src/xpbd.cpp:1167-1369).  One CTA per island (k_solve.cu) follows it
// step for step; an island of tens of thousands of contacts (a settled pile)
// needs every SM, so islands above the giant threshold run here, in one
// cooperative launch whose CTAs meet at a bounded grid barrier between the
// stages the reference separates:
//
//  - colouring: contact p takes the first colour free on both of its dynamic
//    bodies among the contacts before it in island order.  Only the previous
//    contact on each of its two bodies matters (it already folded everything
//    earlier into the body's colour mask), so each contact waits for those two
//    predecessors - found from per-body incidence lists sorted by position -
//    and the colouring runs as a dataflow over the whole grid.  Every thread
//    takes its positions in ascending order; the lowest uncoloured position
//    can always proceed, so the waits end.  Result: the reference's colours.
//  - buckets: a stable counting sort of positions by colour (chunk
//    histograms, one scan, ranked placement), i.e. contact order inside each
//    colour, as the reference regroups them.
//  - the overflow bucket (colour 8), solved serially by the reference, runs
//    on CTA 0 level by level: overflow contacts that share no dynamic body
//    commute, so each level's contacts run at once and every contact sees its
//    bodies exactly as the serial order leaves them.  A contact's level is one
//    above the levels of the previous overflow contact on each of its bodies
//    (found by walking back the body's incidence list); the levels are
//    computed by a grid-wide dataflow like the colouring and the overflow is
//    regrouped by level with a counting sort, so a level's contacts are
//    contiguous.
//  - joints stay serial on one thread, as in the reference.
// Every wait (dataflow or barrier) is bounded; one that runs out raises the
// error word and lets the kernel finish.
#include "m3d_dev.cuh"
#include "m3d_solve.cuh"

namespace m3g
{

// one CTA of 512 threads per SM (128 registers each): the serial overflow
// levels run on CTA 0, and a level of a few hundred contacts takes one pass
constexpr int kGiantThreads = 512;
constexpr int kGiantChunk = kGiantThreads; // positions per colour-histogram chunk
constexpr uint32_t kGiantSpinLimit = 1u << 22;
constexpr uint32_t kNoEnd = 0xFFFFFFFFu;

struct GiantArgs
{
	BodySoA B;
	ContactSoA C;
	JointRec* J;
	const IslandRec* islands;
	const int32_t* giantList;
	const uint32_t* giantDev;
	const uint32_t* bodyVals;
	const uint32_t* contactVals;
	const uint32_t* jointVals;
	uint32_t* colorMask;  // per body: colours taken so far
	uint32_t* localIndex; // per body: index in its island's body list
	uint32_t* bodyOffs;   // per island body + 1: incidence counts, then CSR offsets
	uint32_t* bodyCursor; // per island body: fill cursor, then overflow levels
	uint32_t* incidence;  // 2 per island contact: positions, ascending per body
	int32_t* pred;        // 2 per island contact position: previous position on end A / B; then, per
	                      // position, its overflow index and, per overflow index, its level
	int32_t* ovOrder;     // overflow contacts grouped by level
	uint32_t* levelStart; // per level + 2: offsets into ovOrder
	unsigned long long* done; // per island contact position: epoch << 32 | its bodies' colour masks after it
	                          // (end A << 8 | end B) once coloured
	int32_t* order;       // per island contact position: contact of the bucket order
	int32_t* pmax;        // per position: colour during colouring, then the packet's point count
	int32_t* contactColor;
	uint32_t* chunkHist;  // colour-major chunk histograms, then their offsets
	uint32_t* misc;       // [0..9] bucket starts, [10] colour count, [11] overflow levels
	uint32_t* barrier;    // [0] arrivals, [1] generation, [2] stop: a wait of this launch gave up
	unsigned long long* phaseNs; // [0..5] globaltimer at the ends of the stages of the last island, [8..15]
	                             // time per substep stage summed over the substeps (profiling)
	uint32_t* error;
	uint32_t spinLimit; // unsuccessful polls before a wait gives up
	uint32_t epoch;
	SolveParams P;
};

__device__ __forceinline__ uint32_t ldAcquire(const uint32_t* p) { return *(const volatile uint32_t*)p; }

// stage timestamps of the giant solve, read by m3d_gpu_giant_profile
__device__ __forceinline__ unsigned long long globalNs()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}
__device__ __forceinline__ void stamp(const GiantArgs& a, int k)
{
	if (blockIdx.x == 0 && threadIdx.x == 0)
	{
		a.phaseNs[k] = globalNs();
	}
}
// substep stages: 0 integrate + prepare + packets, 1 coloured normals,
// 2 overflow normals and joints, 3 friction, 4 reconstruct, 5 coloured
// velocity pass, 6 overflow velocity pass and joints
__device__ __forceinline__ void lap(const GiantArgs& a, unsigned long long& t0, int k)
{
	if (blockIdx.x == 0 && threadIdx.x == 0)
	{
		const unsigned long long t = globalNs();
		a.phaseNs[8 + k] += t - t0;
		t0 = t;
	}
}

// island-local index of a contact end that the solve writes (non-zero inverse
// mass) and that belongs to the island's body list; kNoEnd otherwise
__device__ __forceinline__ uint32_t islandEnd(const GiantArgs& a, const uint32_t* bodies, int nb, int body)
{
	if (a.B.massInv[body].x == 0.0f)
	{
		return kNoEnd;
	}
	const uint32_t l = a.localIndex[body];
	return l < (uint32_t)nb && bodies[l] == (uint32_t)body ? l : kNoEnd;
}

// a wait gave up: raise the step's error word and make every CTA stop at its
// next barrier
__device__ __forceinline__ void giveUp(const GiantArgs& a)
{
	atomicOr(&a.barrier[2], 1u);
	atomicOr(a.error, 1u);
}

// All CTAs meet here; writes before it are visible to reads after it.
// Returns true (to every thread of the CTA) when a wait of this launch gave
// up: the caller returns at once, so no stage runs on the partial results of
// the stage before.
__device__ bool gridSync(const GiantArgs& a, uint32_t* gen, uint32_t* stop)
{
	__syncthreads();
	if (threadIdx.x == 0)
	{
		const uint32_t g = *gen;
		__threadfence();
		if (atomicAdd(&a.barrier[0], 1u) == gridDim.x - 1)
		{
			atomicExch(&a.barrier[0], 0u);
			__threadfence();
			atomicExch(&a.barrier[1], g + 1u);
		}
		else
		{
			uint32_t it = 0;
			while (ldAcquire(&a.barrier[1]) == g)
			{
				if (it++ >= a.spinLimit)
				{
					giveUp(a);
					break;
				}
				__nanosleep(32);
			}
		}
		__threadfence();
		*gen = g + 1u;
		*stop = ldAcquire(&a.barrier[2]);
	}
	__syncthreads();
	return *stop != 0u;
}

// exclusive scan of v[0..n) in place by the calling CTA; returns the total
// to every thread of the CTA
__device__ uint32_t ctaScan(uint32_t* v, int n, uint32_t* warpSums)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	uint32_t carry = 0;
	for (int base = 0; base < n; base += kGiantThreads)
	{
		const int i = base + threadIdx.x;
		const uint32_t x = i < n ? v[i] : 0u;
		uint32_t inc = x;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1)
		{
			uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
			if (lane >= o)
			{
				inc += t;
			}
		}
		if (lane == 31)
		{
			warpSums[warp] = inc;
		}
		__syncthreads();
		if (threadIdx.x == 0)
		{
			uint32_t run = 0;
			for (int w = 0; w < kGiantThreads / 32; ++w)
			{
				uint32_t t = warpSums[w];
				warpSums[w] = run;
				run += t;
			}
			warpSums[kGiantThreads / 32] = run;
		}
		__syncthreads();
		if (i < n)
		{
			v[i] = carry + warpSums[warp] + inc - x;
		}
		carry += warpSums[kGiantThreads / 32];
		__syncthreads();
	}
	return carry;
}

enum GiantOp
{
	kGiantNormals,
	kGiantFriction,
	kGiantVelocity
};

__device__ __forceinline__ void giantContactOp(GiantOp op, const GiantArgs& a, int c)
{
	if (op == kGiantNormals)
	{
		solveContactNormalsPrefetched(a.B, a.C, c, a.P.maxCorrection);
	}
	else if (op == kGiantFriction)
	{
		applyContactFrictionPrefetched(a.B, a.C, c);
	}
	else
	{
		solveContactVelocityPrefetched(a.B, a.C, c, a.P.h, a.P.gravityLen);
	}
}

// the overflow bucket in reference order, level by level on CTA 0
// Levels of more than one CTA pass run on the whole grid (one pass and a grid
// barrier instead of several passes of CTA 0); runs of smaller levels run on
// CTA 0 with block barriers, and a grid barrier separates a run from a large
// level after it.  The caller's barrier after the sweep covers the last run.
// Returns true when a wait gave up (the caller returns).
__device__ bool overflowSweep(GiantOp op, const GiantArgs& a, int levels, uint32_t* gen, uint32_t* stop)
{
	const int gtid = blockIdx.x * kGiantThreads + threadIdx.x;
	const int gthreads = gridDim.x * kGiantThreads;
	int L = 1;
	while (L <= levels)
	{
		const int s0 = (int)a.levelStart[L], e0 = (int)a.levelStart[L + 1];
		if (e0 - s0 > kGiantThreads)
		{
			for (int q = s0 + gtid; q < e0; q += gthreads)
			{
				giantContactOp(op, a, a.ovOrder[q]);
			}
			if (gridSync(a, gen, stop))
			{
				return true;
			}
			++L;
			continue;
		}
		int Lend = L;
		while (Lend <= levels && (int)(a.levelStart[Lend + 1] - a.levelStart[Lend]) <= kGiantThreads)
		{
			++Lend;
		}
		if (blockIdx.x == 0)
		{
			for (int l = L; l < Lend; ++l)
			{
				const int e = (int)a.levelStart[l + 1];
				for (int q = (int)a.levelStart[l] + threadIdx.x; q < e; q += kGiantThreads)
				{
					giantContactOp(op, a, a.ovOrder[q]);
				}
				__syncthreads();
			}
		}
		if (Lend <= levels && gridSync(a, gen, stop))
		{
			return true;
		}
		L = Lend;
	}
	return false;
}

// Overflow index of the previous overflow contact on island body `l` before
// island position p, or -1.  `ovIdx` maps island positions to overflow
// indices (-1 for positions with a colour).
__device__ __forceinline__ int32_t overflowPred(const GiantArgs& a, const uint32_t* incidence, const int32_t* ovIdx,
												uint32_t l, uint32_t p)
{
	if (l == kNoEnd)
	{
		return -1;
	}
	const uint32_t s0 = a.bodyOffs[l], s1 = a.bodyOffs[l + 1];
	uint32_t k = s0;
	while (k < s1 && incidence[k] != p)
	{
		++k;
	}
	while (k > s0)
	{
		--k;
		const int32_t i = ovIdx[incidence[k]];
		if (i >= 0)
		{
			return i;
		}
	}
	return -1;
}

__global__ void __launch_bounds__(kGiantThreads, 65536 / (kGiantThreads * 128)) kSolveGiant(GiantArgs a)
{
	__shared__ uint32_t gen, stop;
	__shared__ uint32_t warpSums[kGiantThreads / 32 + 1];
	__shared__ int32_t bucket[kMaxGraphColors + 2];
	__shared__ uint32_t chunkCount[kMaxGraphColors + 1];
	__shared__ uint32_t warpColor[kGiantThreads / 32][kMaxGraphColors + 1];
	if (threadIdx.x == 0)
	{
		gen = ldAcquire(&a.barrier[1]);
	}
	__syncthreads();
	const int gtid = blockIdx.x * kGiantThreads + threadIdx.x;
	const int gthreads = gridDim.x * kGiantThreads;
	const BodySoA& B = a.B;
	const ContactSoA& C = a.C;
	const SolveParams& P = a.P;
	const int islandsHere = (int)*a.giantDev;

	for (int gi = 0; gi < islandsHere; ++gi)
	{
		const IslandRec r = a.islands[a.giantList[gi]];
		const uint32_t* bodies = a.bodyVals + r.bodyStart;
		const uint32_t* contacts = a.contactVals + r.contactStart;
		const uint32_t* joints = a.jointVals + r.jointStart;
		int32_t* order = a.order + r.contactStart;
		int32_t* pmax = a.pmax + r.contactStart;
		int32_t* pred = a.pred + 2 * (int64_t)r.contactStart;
		unsigned long long* done = a.done + r.contactStart;
		uint32_t* incidence = a.incidence + 2 * (int64_t)r.contactStart;
		const int nb = r.bodyCount, nc = r.contactCount;
		int32_t* ovIdx = pred;       // per position, once the colouring is done
		int32_t* ovLevel = pred + nc; // per overflow index
		stamp(a, 0);

		// ---- incidence lists: island contacts per dynamic body, ascending position
		for (int b = gtid; b < nb; b += gthreads)
		{
			const uint32_t body = bodies[b];
			a.localIndex[body] = (uint32_t)b;
			a.colorMask[body] = 0u;
			a.bodyOffs[b] = 0u;
			a.bodyCursor[b] = 0u;
		}
		if (gtid == 0)
		{
			a.bodyOffs[nb] = 0u;
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		for (int p = gtid; p < nc; p += gthreads)
		{
			const int2 ab = C.bodies[contacts[p]];
			pred[2 * p] = -1;
			pred[2 * p + 1] = -1;
			const uint32_t la = islandEnd(a, bodies, nb, ab.x), lb = islandEnd(a, bodies, nb, ab.y);
			if (la != kNoEnd)
			{
				atomicAdd(&a.bodyOffs[la], 1u);
			}
			if (lb != kNoEnd)
			{
				atomicAdd(&a.bodyOffs[lb], 1u);
			}
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		if (blockIdx.x == 0)
		{
			uint32_t total = ctaScan(a.bodyOffs, nb, warpSums);
			if (threadIdx.x == 0)
			{
				a.bodyOffs[nb] = total;
			}
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		for (int p = gtid; p < nc; p += gthreads)
		{
			const int2 ab = C.bodies[contacts[p]];
			const uint32_t la = islandEnd(a, bodies, nb, ab.x), lb = islandEnd(a, bodies, nb, ab.y);
			if (la != kNoEnd)
			{
				incidence[a.bodyOffs[la] + atomicAdd(&a.bodyCursor[la], 1u)] = (uint32_t)p;
			}
			if (lb != kNoEnd)
			{
				incidence[a.bodyOffs[lb] + atomicAdd(&a.bodyCursor[lb], 1u)] = (uint32_t)p;
			}
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		for (int b = gtid; b < nb; b += gthreads)
		{
			const uint32_t s0 = a.bodyOffs[b], s1 = a.bodyOffs[b + 1];
			for (uint32_t i = s0 + 1; i < s1; ++i) // insertion sort: a body has a handful of contacts
			{
				const uint32_t v = incidence[i];
				uint32_t j = i;
				while (j > s0 && incidence[j - 1] > v)
				{
					incidence[j] = incidence[j - 1];
					--j;
				}
				incidence[j] = v;
			}
			const uint32_t body = bodies[b];
			for (uint32_t i = s0 + 1; i < s1; ++i)
			{
				const uint32_t p = incidence[i];
				const int2 ab = C.bodies[contacts[p]];
				pred[2 * p + ((uint32_t)ab.x == body ? 0 : 1)] = (int32_t)incidence[i - 1];
			}
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		stamp(a, 1);

		// ---- greedy first-fit colouring as a dataflow (src/xpbd.cpp:1179-1235)
		// A contact's done word carries its bodies' colour masks after it, so
		// the next contact on a body reads the mask with the flag it waits
		// on (one memory round trip per link of the chain).
		for (int p = gtid; p < nc; p += gthreads)
		{
			const int32_t pa = pred[2 * p], pb = pred[2 * p + 1];
			const int c = (int)contacts[p];
			const int2 ab = C.bodies[c];
			const bool dynA = B.massInv[ab.x].x > 0.0f;
			const bool dynB = B.massInv[ab.y].x > 0.0f;
			// which end of each predecessor is the shared body (static data,
			// read before waiting): 8 = its end A, 0 = its end B
			const int shA = pa >= 0 && C.bodies[contacts[pa]].x == ab.x ? 8 : 0;
			const int shB = pb >= 0 && C.bodies[contacts[pb]].x == ab.y ? 8 : 0;
			unsigned long long wa = 0ull, wb = 0ull;
			for (uint32_t it = 0;; ++it)
			{
				bool ready = true;
				if (pa >= 0)
				{
					wa = *(const volatile unsigned long long*)&done[pa];
					ready = ready && (uint32_t)(wa >> 32) == a.epoch;
				}
				if (pb >= 0)
				{
					wb = *(const volatile unsigned long long*)&done[pb];
					ready = ready && (uint32_t)(wb >> 32) == a.epoch;
				}
				if (ready)
				{
					break;
				}
				if (it >= a.spinLimit)
				{
					giveUp(a);
					break;
				}
				__nanosleep(20);
			}
			const uint32_t ma = dynA && pa >= 0 ? (uint32_t)(wa >> shA) & 0xFFu : 0u;
			const uint32_t mb = dynB && pb >= 0 ? (uint32_t)(wb >> shB) & 0xFFu : 0u;
			const uint32_t freeBits = ~(ma | mb);
			int color = freeBits != 0 ? __ffs((int)freeBits) - 1 : kMaxGraphColors;
			uint32_t na = ma, nb = mb;
			if (color >= kMaxGraphColors)
			{
				color = kMaxGraphColors;
			}
			else
			{
				const uint32_t bit = 1u << color;
				na = dynA ? ma | bit : 0u;
				nb = dynB ? mb | bit : 0u;
			}
			a.contactColor[c] = color;
			pmax[p] = color;
			*(volatile unsigned long long*)&done[p] =
				((unsigned long long)a.epoch << 32) | (unsigned long long)((na << 8) | nb);
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		stamp(a, 2);

		// ---- buckets: stable counting sort of positions by colour
		const int chunks = (nc + kGiantChunk - 1) / kGiantChunk;
		for (int k = blockIdx.x; k < chunks; k += gridDim.x)
		{
			if (threadIdx.x <= kMaxGraphColors)
			{
				chunkCount[threadIdx.x] = 0u;
			}
			__syncthreads();
			const int p = k * kGiantChunk + threadIdx.x;
			if (p < nc)
			{
				atomicAdd(&chunkCount[pmax[p]], 1u);
			}
			__syncthreads();
			if (threadIdx.x <= kMaxGraphColors)
			{
				a.chunkHist[threadIdx.x * chunks + k] = chunkCount[threadIdx.x];
			}
			__syncthreads();
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		if (blockIdx.x == 0)
		{
			ctaScan(a.chunkHist, (kMaxGraphColors + 1) * chunks, warpSums);
			if (threadIdx.x <= kMaxGraphColors)
			{
				a.misc[threadIdx.x] = a.chunkHist[threadIdx.x * chunks];
			}
			if (threadIdx.x == 0)
			{
				a.misc[kMaxGraphColors + 1] = (uint32_t)nc;
			}
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		if (threadIdx.x <= kMaxGraphColors + 1)
		{
			bucket[threadIdx.x] = (int32_t)a.misc[threadIdx.x];
		}
		__syncthreads();
		int ncol = 0;
		for (int c = 0; c < kMaxGraphColors; ++c)
		{
			ncol = bucket[c + 1] > bucket[c] ? c + 1 : ncol;
		}
		for (int k = blockIdx.x; k < chunks; k += gridDim.x)
		{
			const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
			for (int i = threadIdx.x; i < (kGiantThreads / 32) * (kMaxGraphColors + 1); i += kGiantThreads)
			{
				(&warpColor[0][0])[i] = 0u;
			}
			__syncthreads();
			const int p = k * kGiantChunk + threadIdx.x;
			const bool valid = p < nc;
			const int color = valid ? pmax[p] : kMaxGraphColors + 1;
			const uint32_t peers = __match_any_sync(0xffffffffu, color);
			const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
			if (valid && rank == 0)
			{
				warpColor[warp][color] = __popc(peers);
			}
			__syncthreads();
			if (threadIdx.x <= kMaxGraphColors)
			{
				uint32_t run = 0;
				for (int w = 0; w < kGiantThreads / 32; ++w)
				{
					uint32_t t = warpColor[w][threadIdx.x];
					warpColor[w][threadIdx.x] = run;
					run += t;
				}
			}
			__syncthreads();
			if (valid)
			{
				const int q = (int)(a.chunkHist[color * chunks + k] + warpColor[warp][color] + rank);
				order[q] = (int32_t)contacts[p];
				ovIdx[p] = color == kMaxGraphColors ? q - bucket[kMaxGraphColors] : -1;
			}
			__syncthreads();
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		stamp(a, 3);

		// ---- overflow levels (serial order of the overflow bucket)
		const int o0 = bucket[kMaxGraphColors], o1 = bucket[kMaxGraphColors + 1];
		const int nov = o1 - o0;
		if (nov > 0)
		{
			for (int i = gtid; i < nov + 2; i += gthreads)
			{
				a.levelStart[i] = 0u;
				if (i < nov)
				{
					ovLevel[i] = 0;
				}
			}
			if (gtid == 0)
			{
				a.misc[kMaxGraphColors + 3] = 0u;
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
			// dataflow: an overflow contact waits for the levels of its
			// predecessors; every thread takes its indices in ascending order,
			// so the lowest unlevelled index can always proceed
			for (int i = gtid; i < nov; i += gthreads)
			{
				const int c = order[o0 + i];
				const int2 ab = C.bodies[c];
				// island position of overflow index i: the position on the
				// contact's first island body whose overflow index is i
				const uint32_t la = islandEnd(a, bodies, nb, ab.x), lb = islandEnd(a, bodies, nb, ab.y);
				uint32_t p = kNoEnd;
				const uint32_t l0 = la != kNoEnd ? la : lb;
				for (uint32_t k = l0 != kNoEnd ? a.bodyOffs[l0] : 0u; l0 != kNoEnd && k < a.bodyOffs[l0 + 1]; ++k)
				{
					const uint32_t pk = incidence[k];
					if (ovIdx[pk] == i)
					{
						p = pk;
						break;
					}
				}
				const int32_t ia = overflowPred(a, incidence, ovIdx, la, p);
				const int32_t ib = overflowPred(a, incidence, ovIdx, lb, p);
				int32_t lvA = 0, lvB = 0;
				for (uint32_t it = 0;; ++it)
				{
					lvA = ia >= 0 ? *(volatile int32_t*)&ovLevel[ia] : 1;
					lvB = ib >= 0 ? *(volatile int32_t*)&ovLevel[ib] : 1;
					if (lvA != 0 && lvB != 0)
					{
						break;
					}
					if (it >= a.spinLimit)
					{
						giveUp(a);
						lvA = lvA != 0 ? lvA : 1;
						lvB = lvB != 0 ? lvB : 1;
						break;
					}
					__nanosleep(20);
				}
				const int32_t lv = 1 + ((ia >= 0 ? lvA : 0) > (ib >= 0 ? lvB : 0) ? (ia >= 0 ? lvA : 0) : (ib >= 0 ? lvB : 0));
				atomicAdd(&a.levelStart[lv + 1], 1u);
				atomicMax(&a.misc[kMaxGraphColors + 3], (uint32_t)lv);
				__threadfence();
				*(volatile int32_t*)&ovLevel[i] = lv;
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
			if (blockIdx.x == 0)
			{
				const int levels = (int)a.misc[kMaxGraphColors + 3];
				ctaScan(a.levelStart, levels + 2, warpSums);
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
			// placement; the order inside a level does not matter (its
			// contacts share no dynamic body).  Level L's count sat at
			// levelStart[L + 1]; after the exclusive scan that entry holds the
			// level's start and the placement advances it to the level's end,
			// so afterwards level L spans [levelStart[L], levelStart[L + 1]).
			for (int i = gtid; i < nov; i += gthreads)
			{
				const int32_t lv = ovLevel[i];
				a.ovOrder[atomicAdd(&a.levelStart[lv + 1], 1u)] = order[o0 + i];
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
		}
		if (gtid == 0)
		{
			a.misc[kMaxGraphColors + 4] = (uint32_t)nov;
		}
		if (r.jointCount > 0)
		{
			for (int b = gtid; b < nb; b += gthreads)
			{
				refreshInvInertia(B, (int)bodies[b]);
			}
		}
		if (gridSync(a, &gen, &stop))
		{
			return;
		}
		const int overLevels = nov > 0 ? (int)a.misc[kMaxGraphColors + 3] : 0;
		if (r.jointCount > 0)
		{
			if (gtid == 0)
			{
				for (int j = 0; j < r.jointCount; ++j)
				{
					jointPrepare(B, a.J, (int)joints[j]);
				}
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
		}

		stamp(a, 4);

		// ---- substeps (src/xpbd.cpp:1237-1369)
		const int colored = bucket[kMaxGraphColors];
		unsigned long long t0 = 0;
		if (blockIdx.x == 0 && threadIdx.x == 0)
		{
			for (int k = 8; k < 15; ++k)
			{
				a.phaseNs[k] = 0ull;
			}
			t0 = globalNs();
		}
		for (int sub = 0; sub < P.substeps; ++sub)
		{
			for (int b = gtid; b < nb; b += gthreads)
			{
				integrateBody(B, (int)bodies[b], P.h, P.gravity);
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
			for (int p = gtid; p < nc; p += gthreads)
			{
				prepareContact(B, C, (int)contacts[p], P.h);
			}
			if (gtid == 0)
			{
				for (int j = 0; j < r.jointCount; ++j)
				{
					jointReset(a.J, (int)joints[j]);
				}
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
			// packets of 8 consecutive bucket entries share the largest point count
			for (int q = gtid; q < colored; q += gthreads)
			{
				int color = 0;
				while (q >= bucket[color + 1])
				{
					++color;
				}
				const int bs = bucket[color], be = bucket[color + 1];
				const int p0 = bs + ((q - bs) & ~7);
				const int p1 = p0 + 8 < be ? p0 + 8 : be;
				int m = 0;
				for (int p = p0; p < p1; ++p)
				{
					const int pc = C.pointCount[order[p]];
					m = pc > m ? pc : m;
				}
				pmax[q] = m;
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
			lap(a, t0, 0);
			for (int it = 0; it < P.iterations; ++it)
			{
				if (r.jointCount > 0)
				{
					if (gtid == 0)
					{
						for (int j = 0; j < r.jointCount; ++j)
						{
							jointPosition(B, a.J, (int)joints[j], P.h);
						}
					}
					if (gridSync(a, &gen, &stop))
					{
						return;
					}
				}
				for (int color = 0; color < ncol; ++color)
				{
					for (int q = bucket[color] + gtid; q < bucket[color + 1]; q += gthreads)
					{
						solvePacketLane(B, C, order[q], pmax[q], P.maxCorrection);
					}
					if (gridSync(a, &gen, &stop))
					{
						return;
					}
				}
				lap(a, t0, 1);
				if (overLevels > 0)
				{
					if (overflowSweep(kGiantNormals, a, overLevels, &gen, &stop))
					{
						return;
					}
					if (gridSync(a, &gen, &stop))
					{
						return;
					}
				}
				lap(a, t0, 2);
			}
			for (int color = 0; color < ncol; ++color)
			{
				for (int q = bucket[color] + gtid; q < bucket[color + 1]; q += gthreads)
				{
					applyContactFriction(B, C, order[q]);
				}
				if (gridSync(a, &gen, &stop))
				{
					return;
				}
			}
			if (overLevels > 0)
			{
				if (overflowSweep(kGiantFriction, a, overLevels, &gen, &stop))
				{
					return;
				}
				if (gridSync(a, &gen, &stop))
				{
					return;
				}
			}
			lap(a, t0, 3);
			for (int b = gtid; b < nb; b += gthreads)
			{
				reconstructBody(B, (int)bodies[b], P.invH);
			}
			if (gridSync(a, &gen, &stop))
			{
				return;
			}
			lap(a, t0, 4);
			for (int color = 0; color < ncol; ++color)
			{
				for (int q = bucket[color] + gtid; q < bucket[color + 1]; q += gthreads)
				{
					solveContactVelocity(B, C, order[q], P.h, P.gravityLen);
				}
				if (gridSync(a, &gen, &stop))
				{
					return;
				}
			}
			lap(a, t0, 5);
			if (overLevels > 0 || r.jointCount > 0)
			{
				if (overflowSweep(kGiantVelocity, a, overLevels, &gen, &stop))
				{
					return;
				}
				if (gtid == 0)
				{
					for (int j = 0; j < r.jointCount; ++j)
					{
						jointVelocity(B, a.J, (int)joints[j], P.h);
					}
				}
				if (gridSync(a, &gen, &stop))
				{
					return;
				}
			}
			lap(a, t0, 6);
		}
		stamp(a, 5);
	}
}

void launchSolveGiant(DevWorld& w, const SolveParams& P)
{
	if (w.contactMax < w.giantIslandContacts)
	{
		return; // no island can reach the threshold this step
	}
	StepCounters* dc = devCounters(w);
	const size_t nc = (size_t)w.contactMax + 1;
	const size_t nb = (size_t)w.bodyCap + 1;
	const size_t chunks = nc / kGiantChunk + 2;
	w.giantLocal.ensure(nb * sizeof(uint32_t));
	w.giantBodyOffs.ensure((nb + 1) * sizeof(uint32_t));
	w.giantBodyCursor.ensure(nb * sizeof(uint32_t));
	w.giantIncidence.ensure(2 * nc * sizeof(uint32_t));
	w.giantPred.ensure(2 * nc * sizeof(int32_t));
	void* doneBefore = w.giantDone.ptr;
	w.giantDone.ensureZeroed(nc * sizeof(unsigned long long), w.stream);
	w.giantChunkHist.ensure((kMaxGraphColors + 1) * chunks * sizeof(uint32_t));
	w.giantMisc.ensure(16 * sizeof(uint32_t) + 16 * sizeof(unsigned long long));
	w.giantOvOrder.ensure(nc * sizeof(int32_t));
	w.giantLevelStart.ensure((nc + 2) * sizeof(uint32_t));
	w.giantBarrier.ensureZeroed(4 * sizeof(uint32_t), w.stream);
	if (w.giantDone.ptr != doneBefore || ++w.giantEpoch == 0u)
	{
		if (w.giantDone.ptr == doneBefore)
		{
			cudaMemsetAsync(w.giantDone.ptr, 0, w.giantDone.bytes, w.stream);
		}
		w.giantEpoch = 1u;
	}
	if (w.giantGrid == 0)
	{
		int dev = 0, sms = 0, perSm = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kSolveGiant, kGiantThreads, 0);
		perSm = perSm > 2 ? 2 : perSm;
		w.giantGrid = (perSm > 0 ? perSm : 1) * (sms > 0 ? sms : 1);
	}
	GiantArgs a;
	a.B = w.B;
	a.C = w.C;
	a.J = w.joints.as<JointRec>();
	a.islands = w.islands.as<IslandRec>();
	a.giantList = w.giantList.as<int32_t>();
	a.giantDev = &dc->giantIslands;
	a.bodyVals = w.bodyVals.as<uint32_t>();
	a.contactVals = w.contactVals.as<uint32_t>();
	a.jointVals = w.jointVals.as<uint32_t>();
	a.colorMask = w.colorMask.as<uint32_t>();
	a.localIndex = w.giantLocal.as<uint32_t>();
	a.bodyOffs = w.giantBodyOffs.as<uint32_t>();
	a.bodyCursor = w.giantBodyCursor.as<uint32_t>();
	a.incidence = w.giantIncidence.as<uint32_t>();
	a.pred = w.giantPred.as<int32_t>();
	a.ovOrder = w.giantOvOrder.as<int32_t>();
	a.levelStart = w.giantLevelStart.as<uint32_t>();
	a.done = (unsigned long long*)w.giantDone.ptr;
	a.order = w.colorOrder.as<int32_t>();
	a.pmax = w.packetMax.as<int32_t>();
	a.contactColor = w.contactColor.as<int32_t>();
	a.chunkHist = w.giantChunkHist.as<uint32_t>();
	a.misc = w.giantMisc.as<uint32_t>();
	a.barrier = w.giantBarrier.as<uint32_t>();
	a.phaseNs = (unsigned long long*)(w.giantMisc.as<uint32_t>() + 16);
	a.error = &dc->waitErrors;
	a.epoch = w.giantEpoch;
	a.P = P;
	a.spinLimit = w.prim.waitLimit >= 0 ? (uint32_t)(w.prim.waitLimit < 0xFFFFFFFFll ? w.prim.waitLimit : 0xFFFFFFFFll)
										  : kGiantSpinLimit;
	// arrivals and the stop word start from zero even if an earlier launch
	// gave up on a wait (the generation word keeps counting)
	cudaMemsetAsync(w.giantBarrier.ptr, 0, sizeof(uint32_t), w.stream);
	cudaMemsetAsync(w.giantBarrier.as<uint32_t>() + 2, 0, sizeof(uint32_t), w.stream);
	void* args[] = { &a };
	launchBegin("kSolveGiant", w.stream);
	cudaLaunchCooperativeKernel((const void*)kSolveGiant, dim3((unsigned)w.giantGrid), dim3(kGiantThreads), args, 0,
								w.stream);
	launchEnd("kSolveGiant", w.stream);
}

} // namespace m3g

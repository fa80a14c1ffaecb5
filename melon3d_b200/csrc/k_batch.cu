// Batch of worlds in one arena: the two pieces of contact and grid
// bookkeeping that are per world in the reference and global in a single
// arena.
//
//  - Contact order.  Each world's contacts must stay in the order its own
//    contact array has (the solver and the colouring follow it), so the batch
//    keeps contacts world-major: world w's contacts are one block.  A step
//    appends the new pairs after all old contacts (in emission order, which
//    is world-major for grid pairs and again for oversized pairs), then this
//    re-layout gives each world the result of the reference's
//    append-then-swap-remove on its own array A_w = (its old contacts, its new
//    ones in emission order): survivors keep their place, holes below
//    S_w = |A_w| - removed_w take the closed-form sources of the descending
//    swap-remove (see k_broadphase.cu), and the worlds are packed again.  The
//    moved contacts land in the second contact arena, which then becomes the
//    live one.
//  - Stable tier.  The reference rebuilds a world's stable tier on its own
//    schedule.  Worlds that do not rebuild this step keep their entries: they
//    are set aside before the fresh entries of the rebuilding worlds are
//    emitted and appended after them; the tier sort (keys carry the world
//    above the cell) puts every world back in its own key order.
#include "m3d_dev.cuh"

namespace m3g
{

__device__ __forceinline__ uint32_t contactWorld(const BodySoA& B, const ContactSoA& C, int c)
{
	return worldOfBody(B, C.bodies[c].x);
}

// ---- stable tier: entries of worlds that keep their tier --------------------

__global__ void kKeepFlags(const BodySoA B, const uint32_t* vals, int64_t n, const uint8_t* rebuild, uint32_t* flag)
{
	M3G_KERNEL_BEGIN();
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		flag[i] = rebuild[worldOfBody(B, (int)vals[i])] ? 0u : 1u;
	}
}

__global__ void kKeepScatter(const uint64_t* keys, const uint32_t* vals, int64_t n, const uint32_t* flag,
							 const uint32_t* scan, uint64_t* outKeys, uint32_t* outVals, int bits, uint32_t* ranges)
{
	M3G_KERNEL_BEGIN();
	int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n || !flag[i])
	{
		return;
	}
	const uint64_t k = keys[i];
	outKeys[scan[i]] = k;
	outVals[scan[i]] = vals[i];
	const uint64_t mask = (1ull << bits) - 1ull;
	const uint32_t f[4] = { (uint32_t)(k >> (3 * bits)), (uint32_t)((k >> (2 * bits)) & mask),
							(uint32_t)((k >> bits) & mask), (uint32_t)(k & mask) };
	for (int a = 0; a < 4; ++a)
	{
		atomicMin(&ranges[a], f[a]);
		atomicMax(&ranges[4 + a], f[a]);
	}
}

__global__ void kKeepOver(const BodySoA B, const int32_t* over, int32_t n, const uint8_t* rebuild, uint32_t* flag)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
	{
		flag[i] = rebuild[worldOfBody(B, over[i])] ? 0u : 1u;
	}
}

__global__ void kKeepOverScatter(const int32_t* over, int32_t n, const uint32_t* flag, const uint32_t* scan, int32_t* out)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n && flag[i])
	{
		out[scan[i]] = over[i];
	}
}

// Before the stable tier is emitted: set aside the entries (and oversized
// bodies) of the worlds that keep their tier.  Counts go to the step
// counters, the key ranges into the stable tier's slot of `ranges`.
void launchKeepStable(DevWorld& w, uint32_t* ranges)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	const int64_t n = w.stableEntries;
	const int32_t no = w.stableOverCount;
	w.keptKeys.ensure((size_t)(n + 1) * sizeof(uint64_t));
	w.keptVals.ensure((size_t)(n + 1) * sizeof(uint32_t));
	w.keptOver.ensure((size_t)(no + 1) * sizeof(int32_t));
	const int64_t m = n > no ? n : no;
	w.vFlag.ensure((size_t)(m + 2) * sizeof(uint32_t));
	w.vScan.ensure((size_t)(m + 2) * sizeof(uint32_t));
	uint32_t* flag = w.vFlag.as<uint32_t>();
	uint32_t* scan = w.vScan.as<uint32_t>();
	const uint8_t* rebuild = w.worldRebuild.as<uint8_t>();
	if (n > 0)
	{
		M3G_LAUNCH(kKeepFlags, blocksFor(n, 256), 256, s, w.B, w.stableVals.as<uint32_t>(), n, rebuild, flag);
	}
	scanExclusive(flag, scan, n, &dc->keptStable, w.prim, s);
	if (n > 0)
	{
		M3G_LAUNCH(kKeepScatter, blocksFor(n, 256), 256, s, w.stableKeys.as<uint64_t>(), w.stableVals.as<uint32_t>(), n,
				   flag, scan, w.keptKeys.as<uint64_t>(), w.keptVals.as<uint32_t>(), w.keyBits, ranges);
	}
	if (no > 0)
	{
		M3G_LAUNCH(kKeepOver, blocksFor(no, 256), 256, s, w.B, w.stableOver.as<int32_t>(), no, rebuild, flag);
	}
	scanExclusive(flag, scan, no, &dc->keptStableOver, w.prim, s);
	if (no > 0)
	{
		M3G_LAUNCH(kKeepOverScatter, blocksFor(no, 256), 256, s, w.stableOver.as<int32_t>(), no, flag, scan,
				   w.keptOver.as<int32_t>());
	}
}

// merge of two ascending lists of distinct body indices
__global__ void kMergeOver(const int32_t* a, int32_t na, const int32_t* b, int32_t nb, int32_t* out)
{
	M3G_KERNEL_BEGIN();
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < na)
	{
		int32_t lo = 0, hi = nb;
		while (lo < hi)
		{
			int32_t mid = (lo + hi) >> 1;
			if (b[mid] < a[i])
				lo = mid + 1;
			else
				hi = mid;
		}
		out[i + lo] = a[i];
	}
	else if (i < na + nb)
	{
		const int j = i - na;
		int32_t lo = 0, hi = na;
		while (lo < hi)
		{
			int32_t mid = (lo + hi) >> 1;
			if (a[mid] < b[j])
				lo = mid + 1;
			else
				hi = mid;
		}
		out[j + lo] = b[j];
	}
}

// After the first sync: append the kept entries after the fresh ones (the
// caller sorts the tier) and merge the oversized lists.
void launchAppendKeptStable(DevWorld& w, int64_t fresh, int32_t freshOver)
{
	const StepCounters* hc = w.hostCounters;
	cudaStream_t s = w.stream;
	const int64_t kept = hc->keptStable;
	const int32_t keptOver = (int32_t)hc->keptStableOver;
	if (kept > 0)
	{
		cudaMemcpyAsync(w.stableKeys.as<uint64_t>() + fresh, w.keptKeys.ptr, sizeof(uint64_t) * (size_t)kept,
						cudaMemcpyDeviceToDevice, s);
		cudaMemcpyAsync(w.stableVals.as<uint32_t>() + fresh, w.keptVals.ptr, sizeof(uint32_t) * (size_t)kept,
						cudaMemcpyDeviceToDevice, s);
	}
	w.stableEntries = fresh + kept;
	if (keptOver > 0)
	{
		// the merged list goes to scratch first: the fresh list is an input
		w.vSrc.ensure((size_t)(freshOver + keptOver + 1) * sizeof(int32_t));
		M3G_LAUNCH(kMergeOver, blocksFor(freshOver + keptOver, 256), 256, s, w.stableOver.as<int32_t>(), freshOver,
				   w.keptOver.as<int32_t>(), keptOver, w.vSrc.as<int32_t>());
		cudaMemcpyAsync(w.stableOver.ptr, w.vSrc.ptr, sizeof(int32_t) * (size_t)(freshOver + keptOver),
						cudaMemcpyDeviceToDevice, s);
	}
	w.stableOverCount = freshOver + keptOver;
}

// ---- contacts: world-major re-layout ------------------------------------------

// the reference's removal test (src/world.cpp:1705-1735): either body awake
// and the fat boxes no longer overlap
__global__ void kRemovalTest(const BodySoA B, const ContactSoA C, int32_t maxCount, const uint32_t* countDev,
							 uint32_t* removeFlag)
{
	M3G_KERNEL_BEGIN();
	int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= maxCount || c >= (int)*countDev)
	{
		return;
	}
	const int2 ab = C.bodies[c];
	uint32_t rm = 0;
	if ((B.bFlags[ab.x] & kBFAwake) || (B.bFlags[ab.y] & kBFAwake))
	{
		Box a, b;
		a.lo = ld3(B.fatLo[ab.x]);
		a.hi = ld3(B.fatHi[ab.x]);
		b.lo = ld3(B.fatLo[ab.y]);
		b.hi = ld3(B.fatHi[ab.y]);
		rm = overlap(a, b) ? 0u : 1u;
	}
	removeFlag[c] = rm;
}

__global__ void kNewByWorld(const BodySoA B, const ContactSoA C, int32_t maxNew, const uint32_t* newDev, int32_t base,
							uint32_t* wNew, uint64_t* keys, uint32_t* vals)
{
	M3G_KERNEL_BEGIN();
	int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= maxNew || k >= (int)*newDev)
	{
		return;
	}
	const int c = base + k;
	const uint32_t world = contactWorld(B, C, c);
	atomicAdd(&wNew[world], 1u);
	keys[k] = world;
	vals[k] = (uint32_t)c;
}

__global__ void kWorldSizes(const uint32_t* wCount, const uint32_t* wNew, int32_t worlds, uint32_t* wA)
{
	M3G_KERNEL_BEGIN();
	int w = blockIdx.x * blockDim.x + threadIdx.x;
	if (w < worlds)
	{
		wA[w] = wCount[w] + wNew[w];
	}
}

// virtual order: each world's old contacts, then its new ones in emission order
__global__ void kVirtualOrder(const BodySoA B, const ContactSoA C, int32_t oldCount, int32_t maxNew,
							  const uint32_t* newDev, const uint32_t* newByWorld, const uint32_t* wStart,
							  const uint32_t* wCount, const uint32_t* wNewStart, const uint32_t* vStart,
							  const uint32_t* removeFlag, uint32_t* vFlag, uint32_t* vSrc)
{
	M3G_KERNEL_BEGIN();
	int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= oldCount + (int)*newDev)
	{
		vFlag[t] = 0u; // past the live contacts: nothing to scan
		return;
	}
	if (t < oldCount)
	{
		const uint32_t w = contactWorld(B, C, t);
		const uint32_t v = vStart[w] + ((uint32_t)t - wStart[w]);
		vFlag[v] = removeFlag[t];
		vSrc[v] = (uint32_t)t;
	}
	else if (t - oldCount < maxNew && t - oldCount < (int)*newDev)
	{
		const int k = t - oldCount;
		const uint32_t c = newByWorld[k];
		const uint32_t w = contactWorld(B, C, (int)c);
		const uint32_t v = vStart[w] + wCount[w] + ((uint32_t)k - wNewStart[w]);
		vFlag[v] = removeFlag[c];
		vSrc[v] = c;
	}
}

__global__ void kWorldKeep(const uint32_t* wA, const uint32_t* vStart, const uint32_t* vScan, int32_t worlds,
						   uint32_t* wKeep)
{
	M3G_KERNEL_BEGIN();
	int w = blockIdx.x * blockDim.x + threadIdx.x;
	if (w < worlds)
	{
		const uint32_t removed = vScan[vStart[w] + wA[w]] - vScan[vStart[w]];
		wKeep[w] = wA[w] - removed;
	}
}

__device__ void copyContactTo(const ContactSoA& D, int dst, const ContactSoA& S, int src)
{
	D.bodies[dst] = S.bodies[src];
	D.pointCount[dst] = S.pointCount[src];
	D.flags[dst] = S.flags[src];
	D.normal[dst] = S.normal[src];
	D.mat[dst] = S.mat[src];
	D.cachePosA[dst] = S.cachePosA[src];
	D.cacheRotA[dst] = S.cacheRotA[src];
	D.cachePosB[dst] = S.cachePosB[src];
	D.cacheRotB[dst] = S.cacheRotB[src];
	for (int s = 0; s < 4; ++s)
	{
		size_t d = pidx(D, dst, s), o = pidx(S, src, s);
		D.pAnchorA[d] = S.pAnchorA[o];
		D.pAnchorB[d] = S.pAnchorB[o];
		D.pFricA[d] = S.pFricA[o];
		D.pFricB[d] = S.pFricB[o];
		D.pSlip[d] = S.pSlip[o];
		D.pRA[d] = S.pRA[o];
		D.pRB[d] = S.pRB[o];
		D.pJA[d] = S.pJA[o];
		D.pJB[d] = S.pJB[o];
	}
}

// one thread per virtual slot: the world's final position j = its local
// index, when below the world's survivor count
__global__ void kRelayout(const ContactSoA D, const ContactSoA S, const BodySoA B, int32_t total,
						  const uint32_t* totalDev, const uint32_t* vSrc, const uint32_t* vFlag, const uint32_t* vScan,
						  const uint32_t* vStart, const uint32_t* wA, const uint32_t* wKeep,
						  const uint32_t* wFinalStart)
{
	M3G_KERNEL_BEGIN();
	int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= total || t >= (int)*totalDev)
	{
		return;
	}
	const uint32_t w = contactWorld(B, S, (int)vSrc[t]);
	const int32_t base = (int32_t)vStart[w];
	const int32_t j = t - base;
	const int32_t keep = (int32_t)wKeep[w], count = (int32_t)wA[w];
	if (j >= keep)
	{
		return;
	}
	int32_t v = j;
	if (vFlag[t])
	{
		const uint32_t s0 = vScan[base];
		v = keep + (int32_t)(vScan[base + j] - s0);
		for (int guard = 0; guard <= count && v < count && vFlag[base + v]; ++guard)
		{
			v = keep + (int32_t)(vScan[base + v] - s0);
		}
	}
	copyContactTo(D, (int)wFinalStart[w] + j, S, (int)vSrc[base + v]);
}

__global__ void kRelayoutFinish(uint32_t* contactCountDev, const uint32_t* keptTotal, uint32_t* wCount,
								const uint32_t* wKeep, uint32_t* wStart, const uint32_t* wFinalStart, int32_t worlds)
{
	M3G_KERNEL_BEGIN();
	int w = blockIdx.x * blockDim.x + threadIdx.x;
	if (w < worlds)
	{
		wCount[w] = wKeep[w];
		wStart[w] = wFinalStart[w];
	}
	if (w == 0)
	{
		*contactCountDev = *keptTotal;
		wStart[worlds] = *keptTotal;
	}
}

// Replaces the single-world removal: after launchCreateContacts appended the
// new pairs behind the w.contactCount old ones.
void launchBatchRelayout(DevWorld& w)
{
	StepCounters* dc = devCounters(w);
	cudaStream_t s = w.stream;
	const int32_t worlds = w.worldCount;
	const int32_t oldCount = w.contactCount;
	const int32_t maxNew = (int32_t)w.pairTotal;
	const int32_t M = w.contactMax; // old + new upper bound
	const size_t w4 = (size_t)(worlds + 2) * sizeof(uint32_t);
	const size_t c4 = (size_t)(M + 2) * sizeof(uint32_t);
	w.worldNewCount.ensure(w4);
	w.worldNewStart.ensure(w4);
	w.worldVStart.ensure(w4);
	w.worldRemoved.ensure(w4);
	w.worldFinalStart.ensure(w4);
	w.removeFlag.ensure(c4);
	w.removeScan.ensure(c4);
	w.evEndFlag.ensure(c4);
	w.evBeginFlag.ensure(c4);
	w.evRemoval.ensure((size_t)(M + 1) * sizeof(int4));
	w.vFlag.ensure(c4);
	w.vScan.ensure(c4);
	w.vSrc.ensure(c4);
	w.newByWorldKeys.ensure((size_t)(maxNew + 1) * sizeof(uint64_t));
	w.newByWorldVals.ensure((size_t)(maxNew + 1) * sizeof(uint32_t));
	uint32_t* wNew = w.worldNewCount.as<uint32_t>();
	uint32_t* wA = w.worldRemoved.as<uint32_t>(); // |A_w|: old + new contacts of each world
	fillWords(wNew, 0u, w4, s);
	if (maxNew > 0)
	{
		M3G_LAUNCH(kNewByWorld, blocksFor(maxNew, 256), 256, s, w.B, w.C, maxNew, &dc->newContacts, oldCount, wNew,
				   w.newByWorldKeys.as<uint64_t>(), w.newByWorldVals.as<uint32_t>());
		uint64_t worldMask = 0;
		while (worldMask < (uint64_t)(worlds - 1))
		{
			worldMask = (worldMask << 1) | 1ull;
		}
		radixSortPairs(w.newByWorldKeys.as<uint64_t>(), w.newByWorldVals.as<uint32_t>(), maxNew, worldMask, w.prim, s,
					   &dc->newContacts);
	}
	scanExclusive(wNew, w.worldNewStart.as<uint32_t>(), worlds, nullptr, w.prim, s);
	M3G_LAUNCH(kWorldSizes, blocksFor(worlds, 256), 256, s, w.worldContactCount.as<uint32_t>(), wNew, worlds, wA);
	scanExclusive(wA, w.worldVStart.as<uint32_t>(), worlds, w.worldVStart.as<uint32_t>() + worlds, w.prim, s);
	// removal flags over old + new contacts
	const int32_t total = oldCount + maxNew;
	if (total > 0)
	{
		M3G_LAUNCH(kRemovalTest, blocksFor(total, 256), 256, s, w.B, w.C, total, &dc->contactCount,
				   w.removeFlag.as<uint32_t>());
	}
	{
		M3G_LAUNCH(kVirtualOrder, blocksFor(total + 1, 256), 256, s, w.B, w.C, oldCount, maxNew, &dc->newContacts,
				   w.newByWorldVals.as<uint32_t>(), w.worldContactStart.as<uint32_t>(),
				   w.worldContactCount.as<uint32_t>(), w.worldNewStart.as<uint32_t>(), w.worldVStart.as<uint32_t>(),
				   w.removeFlag.as<uint32_t>(), w.vFlag.as<uint32_t>(), w.vSrc.as<uint32_t>());
	}
	// vScan over contactCount + 1 entries: entry V is the total removed
	scanExclusive(w.vFlag.as<uint32_t>(), w.vScan.as<uint32_t>(), total + 1, &dc->removed, w.prim, s);
	uint32_t* keepW = w.worldNewStart.as<uint32_t>(); // the new starts are consumed by kVirtualOrder
	M3G_LAUNCH(kWorldKeep, blocksFor(worlds, 256), 256, s, wA, w.worldVStart.as<uint32_t>(), w.vScan.as<uint32_t>(),
			   worlds, keepW);
	scanExclusive(keepW, w.worldFinalStart.as<uint32_t>(), worlds, &dc->keptContacts, w.prim, s);
	if (total > 0)
	{
		M3G_LAUNCH(kRelayout, blocksFor(total, 256), 256, s, w.C2, w.C, w.B, total, &dc->contactCount,
				   w.vSrc.as<uint32_t>(), w.vFlag.as<uint32_t>(), w.vScan.as<uint32_t>(), w.worldVStart.as<uint32_t>(),
				   wA, keepW, w.worldFinalStart.as<uint32_t>());
	}
	M3G_LAUNCH(kRelayoutFinish, blocksFor(worlds, 256), 256, s, &dc->contactCount, &dc->keptContacts,
			   w.worldContactCount.as<uint32_t>(), keepW, w.worldContactStart.as<uint32_t>(),
			   w.worldFinalStart.as<uint32_t>(), worlds);
	ContactSoA t = w.C;
	w.C = w.C2;
	w.C2 = t;
	setDeviceCount(w, &dc->endRemoval, 0u);
}

} // namespace m3g

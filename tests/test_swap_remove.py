"""The contact-removal rule used by the removal kernel (k_broadphase.cu,
kRemovalMoves) against a direct simulation of the reference's descending
swap-remove loop (reference src/world.cpp:100-119, 1722-1734) on random
removal patterns.  The kernel's arithmetic is the same expression; the GPU
parity tests cover the kernel itself."""
import random


def reference_loop(items, removed):
    a = list(items)
    for i in range(len(a) - 1, -1, -1):
        if removed[i]:
            last = len(a) - 1
            if i != last:
                a[i] = a[last]
            a.pop()
    return a


def closed_form(items, removed):
    count = len(items)
    scan, acc = [], 0
    for r in removed:
        scan.append(acc)
        acc += 1 if r else 0
    S = count - acc
    out = list(items[:S])
    for i in range(S):
        if removed[i]:
            p = S + scan[i]
            while p < count and removed[p]:
                p = S + scan[p]
            out[i] = items[p]
    return out


def test_closed_form_matches_reference_loop():
    rng = random.Random(7)
    for trial in range(3000):
        n = rng.randint(0, 40)
        density = rng.random()
        removed = [rng.random() < density for _ in range(n)]
        items = list(range(n))
        assert closed_form(items, removed) == reference_loop(items, removed), (removed,)


def test_tail_removal_case_from_rain():
    # 47 old contacts + 6 new; removed: holes 17,21,24,30,33,36 and old tail 46
    n = 53
    removed = [i in (17, 21, 24, 30, 33, 36, 46) for i in range(n)]
    out = closed_form(list(range(n)), removed)
    assert [out[i] for i in (17, 21, 24, 30, 33, 36)] == [52, 47, 48, 49, 50, 51]

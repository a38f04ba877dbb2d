"""CPU check of the bulge chase's hand-off between sweeps (cuev_b200/csrc/bulge.cu,
bc_chase_kernel).

Model: hop (s, h) has cq, r0 and r1 = min(r1u, n - 1) (r1u = s + b for hop 0, c + 2b - 1 for
hop c = s + 1 + (h - 1) b); its window rows are [cq, hi = min(n - 1, r1 + b)].  It reads the
lower-stored elements {(max(a, c), min(a, c)) : a in [cq, hi], c in [r0, r1]} when it gathers its
strip, writes its beta element (r0, cq) and then publishes prog_ref[s] = cq, writes the rest of the
strip, and publishes prog[s] = cq; hops of one sweep run in order, and the end of a sweep sets both
counters to INT_MAX.  Hop (s, h) starts once prog[s-1] >= need - 1 and prog_ref[s-1] >= need,
need = r1u - b + 1 (the counters start at -1).  The sequential algorithm (the oracle's chase, the
reference's order) finishes sweep s - 1 before sweep s starts, so every pair of hops of different
sweeps whose footprints overlap must be ordered, directly or through earlier waits: the earlier hop
complete before the later one gathers, or, when the overlap is only the earlier hop's beta element,
that element written.  The check runs over sizes around the band width; the same model with the
thresholds taken from the clipped r1 (an earlier form of the kernel) must show races for n <= b.
"""
import pytest


def _hops(n, b):
    sweeps = []
    for s in range(n - 2):
        hl, hop = [], 0
        while True:
            if hop == 0:
                cq, r0, r1u = s, s + 1, s + b
            else:
                c = s + 1 + (hop - 1) * b
                if c + b >= n:
                    break
                cq, r0, r1u = c, c + b, c + 2 * b - 1
            r1 = min(r1u, n - 1)
            hl.append((cq, r0, r1, r1u, min(n - 1, r1 + b)))
            hop += 1
        sweeps.append(hl)
    return sweeps


def _races(n, b, clipped=False):
    H = _hops(n, b)
    order = [(s, h) for s, hl in enumerate(H) for h in range(len(hl))]
    idx = {sh: i for i, sh in enumerate(order)}
    fp = [{(max(a, c), min(a, c)) for a in range(H[s][h][0], H[s][h][4] + 1)
           for c in range(H[s][h][1], H[s][h][2] + 1)} for s, h in order]
    done = [0] * len(order)   # bitset: hops complete before this hop gathers
    past2 = [0] * len(order)  # bitset: hops whose beta is written before this hop gathers

    def after(i):
        return done[i] | (1 << i), past2[i] | done[i] | (1 << i)

    for q, (s, h) in enumerate(order):
        d = p2 = 0
        if h > 0:
            dd, pp = after(idx[(s, h - 1)])
            d, p2 = d | dd, p2 | pp
        if s > 0:
            _, _, r1, r1u, _ = H[s][h]
            need = (r1 if clipped else r1u) - b + 1
            prev = H[s - 1]
            last = len(prev) - 1
            if need - 1 > -1:  # else the initial -1 already satisfies the wait
                k = next((i for i, x in enumerate(prev) if x[0] >= need - 1), last)
                dd, pp = after(idx[(s - 1, k)])
                d, p2 = d | dd, p2 | pp
            if need > -1:
                k2 = next((i for i, x in enumerate(prev) if x[0] >= need), None)
                if k2 is None:
                    dd, pp = after(idx[(s - 1, last)])
                    d, p2 = d | dd, p2 | pp
                else:
                    r = idx[(s - 1, k2)]
                    p2 |= (1 << r) | past2[r] | done[r]  # started (its wait held), beta written
                    d |= done[r]
                    if k2 > 0:
                        dd, pp = after(idx[(s - 1, k2 - 1)])
                        d, p2 = d | dd, p2 | pp
        done[q], past2[q] = d, p2 | d
    races = []
    for q, (s, h) in enumerate(order):
        cq, hi = H[s][h][0], H[s][h][4]
        for p in range(q):
            ps, ph = order[p]
            if ps >= s or H[ps][ph][4] < cq or hi < H[ps][ph][0]:
                continue
            ov = fp[p] & fp[q]
            if not ov or (done[q] >> p) & 1:
                continue
            pc, pr0 = H[ps][ph][0], H[ps][ph][1]
            if ov <= {(pr0, pc)} and (past2[q] >> p) & 1:
                continue
            races.append(((ps, ph), (s, h)))
    return races


@pytest.mark.parametrize("b", [32, 64])
@pytest.mark.parametrize("n", [10, 33, 40, 65, 70, 100])
def test_chase_waits_order_every_conflicting_pair(n, b):
    assert _races(n, b) == []


@pytest.mark.parametrize("n,b", [(20, 32), (40, 64)])
def test_clipped_thresholds_would_race(n, b):
    assert _races(n, b, clipped=True)

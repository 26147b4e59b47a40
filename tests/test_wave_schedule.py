"""CPU model of the triangular sweeps' schedule (dplasma_b200/csrc/wave_kernel.cu,
trsm_wave_kernel): for every CTA the order in which the producer warp streams
W / M / L blocks into the ring must equal the order in which the consumer
warps take them; every block must receive its products in solve order, then
its Z = W acc, then Y = Z - M Y_prev, then its publish; and the CTAs, each
running its program in order with a flag wait before every remote Y, must
all finish (no cycle of waits).  The model restates the kernel's control flow
(the owner of the block after next applies that block's product and forms
its Z when Y_q arrives and defers its other products past its own publish)."""
import pytest

RMAX = 4


def blk(qi, P, T):
    return P - 1 - qi if T else qi


def pos(p, P, T):
    return P - 1 - p if T else p


def later(p, q, T):
    return p < q if T else p > q


def producer(c, G, P, T):
    out = []
    owned = [c + i * G for i in range(RMAX) if c + i * G < P]
    first = blk(0, P, T)
    if first % G == c:
        out.append(("W", first))
    if P > 1 and blk(1, P, T) % G == c:
        out.append(("W", blk(1, P, T)))
    for qi in range(P):
        q = blk(qi, P, T)
        nq = blk(qi + 1, P, T) if qi + 1 < P else -1
        nnq = blk(qi + 2, P, T) if qi + 2 < P else -1
        if not any(later(p, q, T) for p in owned):
            continue
        if nq >= 0 and nq % G == c:
            out.append(("M", nq))
            if qi >= 1:
                pq = blk(qi - 1, P, T)
                out += [("L", p, pq) for p in owned if pos(p, P, T) > qi + 1]
        if nnq >= 0 and nnq % G == c:
            out += [("L", nnq, q), ("W", nnq)]
        else:
            out += [("L", p, q) for p in owned if p != nq and later(p, q, T)]
    return out


def consumer(c, G, P, T):
    out = []
    owned = [c + i * G for i in range(RMAX) if c + i * G < P]
    first = blk(0, P, T)
    if first % G == c:
        out += [("W", first), ("PUB", first)]
    if P > 1 and blk(1, P, T) % G == c:
        out.append(("W", blk(1, P, T)))
    for qi in range(P):
        q = blk(qi, P, T)
        nq = blk(qi + 1, P, T) if qi + 1 < P else -1
        nnq = blk(qi + 2, P, T) if qi + 2 < P else -1
        if not any(later(p, q, T) for p in owned):
            continue
        if q % G != c:
            out.append(("WAIT", q))
        if nq >= 0 and nq % G == c:
            out += [("M", nq), ("PUB", nq)]
            if qi >= 1:
                pq = blk(qi - 1, P, T)
                out += [("L", p, pq) for p in owned if pos(p, P, T) > qi + 1]
        if nnq >= 0 and nnq % G == c:
            out += [("L", nnq, q), ("W", nnq)]
        else:
            out += [("L", p, q) for p in owned if p != nq and later(p, q, T)]
    return out


def check(G, P, T):
    seqs = {c: consumer(c, G, P, T) for c in range(G)}
    for c in range(G):
        assert producer(c, G, P, T) == [x for x in seqs[c] if x[0] in ("W", "M", "L")], (G, P, T, c)
    for c in range(G):
        hist = {}
        for x in seqs[c]:
            if x[0] != "WAIT":
                hist.setdefault(x[1], []).append(x)
        for b, h in hist.items():
            pb = pos(b, P, T)
            assert [x[2] for x in h if x[0] == "L"] == [blk(j, P, T) for j in range(pb - 1)], (G, P, T, b)
            kinds = [x[0] for x in h if x[0] != "L"]
            assert kinds == (["W", "PUB"] if pb == 0 else ["W", "M", "PUB"]), (G, P, T, b, kinds)
            iw = [i for i, x in enumerate(h) if x[0] == "W"][0]
            assert all(x[0] != "L" for x in h[iw:]), (G, P, T, b)
    pub, ptr, progress = set(), {c: 0 for c in range(G)}, True
    while progress:
        progress = False
        for c in range(G):
            s = seqs[c]
            while ptr[c] < len(s):
                x = s[ptr[c]]
                if x[0] == "WAIT" and x[1] not in pub:
                    break
                if x[0] == "L":
                    assert x[2] in pub
                if x[0] == "M":
                    assert blk(pos(x[1], P, T) - 1, P, T) in pub
                if x[0] == "PUB":
                    pub.add(x[1])
                ptr[c] += 1
                progress = True
    assert all(ptr[c] == len(seqs[c]) for c in range(G)), (G, P, T)
    assert len(pub) == P


@pytest.mark.parametrize("T", [False, True])
@pytest.mark.parametrize("G", range(2, 12))
def test_wave_schedule_small_grids(G, T):
    for P in range(1, RMAX * G + 1):
        check(G, P, T)


@pytest.mark.parametrize("T", [False, True])
@pytest.mark.parametrize("P", [64, 512, 592])
def test_wave_schedule_b200_grid(P, T):
    check(148, P, T)

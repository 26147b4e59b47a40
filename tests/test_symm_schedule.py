"""CPU model of the residual kernel's pipeline (dplasma_b200/csrc/refine.cu,
symm_stream_kernel): one producer warp fills a ring of panel stages and the x
slices; four y_m warps consume every panel, four y_n warps the panels p = w
(mod 4) of each tile after waiting for the tile's x slice.  The model runs all
nine agents in every interleaving order it tries (round-robin with different
priorities) and checks that they all finish (no cycle of waits) and that the
producer never overwrites a buffer still in use: a ring stage before its five
users released it, the x slice of tile t (buffer t mod 2) before every y_n warp
left tile t - 2, the column's x slice before the y_m warps released the
previous column."""
import itertools

import pytest

NP, NST = 32, 7          # panels per tile, ring stages (SY_NP, SY_NST)


def tiles_of(mt, t0, t1):
    """(m, n) of the lower tiles with storage index in [t0, t1) (column order)."""
    out, t = [], 0
    for n in range(mt):
        for m in range(n, mt):
            if t0 <= t < t1:
                out.append((m, n))
            t += 1
    return out


def simulate(mt, t0, t1, order):
    tiles = tiles_of(mt, t0, t1)
    T = len(tiles)
    state = {"filled": {}, "released": {}, "xfull": set(), "xn_free": 0}
    # producer program counter: (tile, panel) with a "x" pseudo-step per tile
    prog = {"P": 0}
    ym = {w: 0 for w in range(4)}             # next global panel index
    yn = {w: (0, 0) for w in range(4)}        # (tile, k-th own panel) ; k = 0..7
    yn_xwait = {w: True for w in range(4)}
    cols_done = 0

    def pidx(t, p):
        return t * NP + p

    # producer step list
    steps = []
    cur_n = None
    for t, (m, n) in enumerate(tiles):
        new_col = n != cur_n
        if new_col and cur_n is not None:
            steps.append(("xn_wait", t))
        steps.append(("x", t))
        for p in range(NP):
            steps.append(("panel", t, p))
        cur_n = n

    def users(i):
        return 5

    def step_producer():
        nonlocal cols_done
        i = prog["P"]
        if i >= len(steps):
            return False
        s = steps[i]
        if s[0] == "xn_wait":
            need = 4 * (cols_done + 1)
            if state["xn_free"] < need:
                return False
            cols_done += 1
        elif s[0] == "x":
            t = s[1]
            # buffer t % 2: every y_n warp has left tile t - 2
            for w in range(4):
                assert yn[w][0] >= t - 1, ("x slice overwritten in use", t, w, yn[w])
            state["xfull"].add(t)
        else:
            t, p = s[1], s[2]
            g = pidx(t, p)
            if g >= NST and state["released"].get(g - NST, 0) < users(g - NST):
                return False
            state["filled"][g] = True
        prog["P"] += 1
        return True

    def step_ym(w):
        g = ym[w]
        if g >= T * NP:
            return False
        if g not in state["filled"]:
            return False
        state["released"][g] = state["released"].get(g, 0) + 1
        ym[w] = g + 1
        t, p = divmod(g, NP)
        if p == NP - 1:
            m, n = tiles[t]
            if m + 1 == mt:
                state["xn_free"] += 1
        return True

    def step_yn(w):
        t, k = yn[w]
        if t >= T:
            return False
        if yn_xwait[w]:
            if t not in state["xfull"]:
                return False
            yn_xwait[w] = False
            return True
        g = pidx(t, w + 4 * k)
        if g not in state["filled"]:
            return False
        state["released"][g] = state["released"].get(g, 0) + 1
        k += 1
        if k == NP // 4:
            yn[w] = (t + 1, 0)
            yn_xwait[w] = True
        else:
            yn[w] = (t, k)
        return True

    agents = [("P", None)] + [("M", w) for w in range(4)] + [("N", w) for w in range(4)]
    agents = [agents[i] for i in order]
    progress = True
    while progress:
        progress = False
        for kind, w in agents:
            while True:
                ok = step_producer() if kind == "P" else (step_ym(w) if kind == "M" else step_yn(w))
                if not ok:
                    break
                progress = True
                if kind != "P":
                    break          # consumers advance one step per turn
    assert prog["P"] == len(steps), ("producer stuck", prog["P"], len(steps))
    assert all(ym[w] == T * NP for w in range(4)), ym
    assert all(yn[w][0] == T for w in range(4)), yn
    # every stage was released by its five users
    assert all(state["released"].get(g, 0) == 5 for g in range(T * NP))


@pytest.mark.parametrize("mt,t0,t1", [(4, 0, 10), (6, 3, 17), (9, 0, 45), (9, 20, 21), (12, 5, 60)])
def test_symm_pipeline_interleavings(mt, t0, t1):
    base = list(range(9))
    orders = [base, base[::-1], [4, 3, 2, 1, 0, 8, 7, 6, 5], [8, 0, 7, 1, 6, 2, 5, 3, 4]]
    orders += [list(p) for p in itertools.islice(itertools.permutations(base), 0, 200, 37)]
    for order in orders:
        simulate(mt, t0, t1, order)

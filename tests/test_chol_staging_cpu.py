"""The staging schedule of the mixed form's blocked Cholesky update
(Block::chol_update_bulk in bdsim_b200/csrc/integrator.cuh), replayed on the
CPU for every factor size the kernel meets.

The kernel keeps three shared-memory buffers of panel rows tagged by their
first row; warp 0 fills a buffer by bulk copies (a "full" mbarrier) only after
every warp has released it (an "empty" mbarrier), and a buffer is released,
and gives up its tag, after the last tile that uses it. These tests restate
the pool's choices and check the invariants the mbarriers rely on: each fill
follows a release of the buffer's previous contents, each tile finds its A
and B rows, no buffer is read after its release, and every copy stays inside
the factor's column and on 16-byte boundaries."""
import pytest

TILE, STRIDE, BUFS, SLOTS, FIRST_SLOT, MAX_BLOCK, MAX_PANEL = 64, 68, 3, 16, 7, 64, 32


def chol_ld(n):
    return (n + 15) // 16 * 16


def update_calls(n, nb):
    """(k0, k1, r0, c0, c1) of every chol_update call of cholesky_blocked."""
    calls, kb = [], 0
    while kb < n:
        ke = min(kb + nb, n)
        for p0 in range(kb, ke, MAX_PANEL):
            if p0 > kb:
                calls.append((kb, p0, p0, p0, min(p0 + MAX_PANEL, ke)))
        if ke >= n:
            break
        calls.append((kb, ke, ke, ke, n))
        kb += nb
    return calls


def replay(n, n_max):
    nvs = (n_max + 7) // 8 * 8
    stage_cap = (SLOTS - FIRST_SLOT) * nvs
    nb = min(stage_cap // (2 * STRIDE), MAX_BLOCK) & ~7
    if n < 300 or nb < 8:
        return 0
    ldl, region = chol_ld(n), n_max * chol_ld(n_max)
    tiles_done = 0
    for k0, k1, r0, c0, c1 in update_calls(n, nb):
        kk = k1 - k0
        kk4 = (kk + 3) & ~3
        if not (BUFS * kk4 * STRIDE + 8 <= stage_cap and r0 % 8 == 0 and c0 % 8 == 0):
            continue
        nti, ntj = -(-(n - r0) // TILE), -(-(c1 - c0) // TILE)
        nt = nti * ntj

        def next_tile(t):
            while t < nt and r0 + (t // ntj) * TILE + TILE - 1 < c0 + (t % ntj) * TILE:
                t += 1
            return t

        tag, pend, held = [-1] * BUFS, [False] * BUFS, [None] * BUFS
        events = [[] for _ in range(BUFS)]

        def find(x):
            f = -1
            for b in range(BUFS):
                if tag[b] == x:
                    f = b
            return f

        def request(x, keep):
            if find(x) >= 0:
                return
            f = -1
            for b in range(BUFS - 1, -1, -1):
                if tag[b] not in keep:
                    f = b
            if f < 0:
                return
            assert not pend[f]
            assert not events[f] or events[f][-1] == "release", "refill before every warp released the buffer"
            cnt = min(TILE, ldl - x)
            assert x % 8 == 0 and cnt > 0 and (cnt * 8) % 16 == 0 and cnt <= STRIDE
            for k in range(kk):
                src = (k0 + k) * ldl + x
                assert src % 2 == 0 and x + cnt <= ldl and src + cnt <= region
            assert (f + 1) * kk4 * STRIDE <= stage_cap - 8
            tag[f], pend[f], held[f] = x, True, x
            events[f].append("fill")

        t = next_tile(0)
        while t < nt:
            i0, j0 = r0 + (t // ntj) * TILE, c0 + (t % ntj) * TILE
            request(i0, (i0, j0, -2))
            request(j0, (i0, j0, -2))
            ba, bb = find(i0), find(j0)
            assert ba >= 0 and bb >= 0 and held[ba] == i0 and held[bb] == j0
            for b in {ba, bb}:
                pend[b] = False
                events[b].append("use")
            tn = next_tile(t + 1)
            i1 = r0 + (tn // ntj) * TILE if tn < nt else -2
            j1 = c0 + (tn % ntj) * TILE if tn < nt else -2
            if tn < nt:
                request(i1, (i0, j0, -2))
                request(j1, (i0, j0, i1))
            for b in {ba, bb}:
                if tag[b] not in (i1, j1):
                    events[b].append("release")
                    tag[b] = -1
            tiles_done += 1
            t = tn
        assert not any(pend), "a fill left pending at the end of the update"
        for ev in events:
            seq = " ".join(ev)
            assert "release use" not in seq and "release release" not in seq and "fill fill" not in seq
    return tiles_done


# The bulk path runs where three staging buffers fit the free vector slots: the
# 32-column sub-panel updates from 3N ~ 727, the 64-column trailing updates from
# 3N ~ 1450 (cfg5, N = 500); smaller factors keep the per-thread staging.
@pytest.mark.parametrize("n_max", [729, 750, 999, 1002, 1200, 1449, 1452, 1500, 1536])
def test_staging_schedule(n_max):
    total = 0
    for n in sorted({300, 729, n_max - 3, n_max}):
        if 300 <= n <= n_max:
            total += replay(n, n_max)
    assert total > 0

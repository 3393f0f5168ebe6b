"""The step schedule of the two-column sweep with an item's passes back to back (`sweep2_item` in
hyalite_b200/csrc/scan_kernel.cuh), restated step by step on the CPU: G lanes, W column pairs a
pass, n passes. Pass p begins with G - 1 transition steps (lane L <= t at column pair t - L of pass
p, the others at W + t - L of pass p - 1), a warp barrier before them and a block barrier after
them; its interior steps s = G - 1 .. W - 1 put lane L at column pair s - L; the last pass ends
with G - 1 drain steps. The checks are the invariants the kernel's correctness rests on:

* every lane visits every (pass, column pair) exactly once, in order;
* lane L works a column pair one step after lane L - 1 did (the shuffle hand-off);
* a lane's state is reset for pass p after its last column of pass p - 1 and before its first of p;
* lane 0 reads pass p's boundary value of column pair c (written by lane G - 1 in pass p - 1) at
  least one step after the write and with a barrier in between, and before lane G - 1 overwrites
  it in pass p (the one-step-ahead loads of the interior read one step early).

The kernel sizes W at least 2G; the boundary ordering fails below 2G - 2, which is why."""
import pytest


def schedule(G, W, n_passes):
    """Returns visits[L] = [(pass, c, step)], resets[L] = [(pass, step)] and barrier steps."""
    visits = {L: [] for L in range(G)}
    resets = {L: [] for L in range(G)}
    barriers = []
    step = 0

    def checked(L, lp, c):
        if lp >= 0 and c >= 0:
            visits[L].append((lp, c, step))

    for ps in range(n_passes):
        barriers.append(step)  # warp barrier before the transition
        for t in range(G - 1):
            for L in range(G):
                fresh = L <= t
                if fresh and L == t and ps > 0:
                    resets[L].append((ps, step))
                checked(L, ps if fresh else ps - 1, t - L if fresh else W + t - L)
            step += 1
        if ps > 0:
            resets[G - 1].append((ps, step))
        barriers.append(step)  # block barrier after the transition
        for s in range(G - 1, W):
            for L in range(G):
                checked(L, ps, s - L)
            step += 1
    for t in range(G - 1):
        for L in range(G):
            checked(L, n_passes - 1 if L > t else -1, W + t - L)
        step += 1
    return visits, resets, barriers


def check_schedule(G, W, n_passes):
    visits, resets, barriers = schedule(G, W, n_passes)
    want = [(p, c) for p in range(n_passes) for c in range(W)]
    at = {}
    for L in range(G):
        assert [(p, c) for p, c, _ in visits[L]] == want, (G, W, n_passes, L)
        for p, c, s in visits[L]:
            at[(L, p, c)] = s
    for L in range(1, G):
        for p, c, s in visits[L]:
            assert at[(L - 1, p, c)] == s - 1, (L, p, c)
    for L in range(G):
        for p, s in resets[L]:
            assert at[(L, p - 1, W - 1)] < s <= at[(L, p, 0)], (L, p)
    for p in range(1, n_passes):
        for c in range(W):
            written = at[(G - 1, p - 1, c)]
            read = at[(0, p, c)] - (1 if c >= G else 0)
            assert read - written >= 1, (p, c)
            assert any(written < b <= read for b in barriers), (p, c)
            assert at[(G - 1, p, c)] > read, (p, c)


@pytest.mark.parametrize("G", [2, 4, 8])
def test_two_column_pass_schedule(G):
    for W in range(2 * G, 2 * G + 40):
        for n in range(1, 6):
            check_schedule(G, W, n)


def test_narrow_passes_break_the_boundary_ordering():
    # From G to 2G - 3 column pairs a pass, the transition reads a boundary value that lane G - 1
    # wrote after the warp barrier; 2G - 2 is the least width the ordering holds at (the kernel
    # pads passes to 2G).
    G = 8
    for W in range(G, 2 * G - 2):
        with pytest.raises(AssertionError):
            check_schedule(G, W, 3)
    check_schedule(G, 2 * G - 2, 3)

"""Index arithmetic of tensor-core and stage-2 kernels, checked on the host
(no GPU).

FP16 SYR2K (`tc_syr2k_tma_kernel`, evd4sc2025_b200/csrc/lowprec.cu): the
packed operand H has n rows of L = 2 kp halves (kp = k rounded up to 64);
chunk t of the left operand [A | B] is the TMA box at x = 64 t, of the right
operand [B | A] at x = (64 t + kp) mod L; boxes are 64 halves (128 bytes)
wide, so x * 2 bytes must be a multiple of 16 and a box must not run past L.
The CTAs walk the lower 128 x 256 tiles of C: column block bn holds tile
rows 2 bn .. tm - 1; every element on or below the diagonal must lie in
exactly one of them.
"""

GM, GN, GK = 128, 256, 64


def g_tile(t, tm):
    c = 0
    while True:
        cnt = tm - 2 * c
        if t < cnt:
            return 2 * c + t, c
        t -= cnt
        c += 1


def test_syr2k_boxes_are_aligned_and_inside_the_row():
    for k in (1, 7, 8, 63, 64, 65, 100, 1024, 1000):
        kp = (k + 63) // 64 * 64
        L = 2 * kp
        for t in range(L // GK):
            for x in (t * GK, (t * GK + kp) % L):
                assert (x * 2) % 16 == 0 and x + GK <= L
        # the row pitch of the tensor map (L halves) is a multiple of 16 bytes
        assert (L * 2) % 16 == 0


def test_syr2k_lower_tiles_cover_the_triangle_once():
    for n in (1, 100, 128, 129, 300, 513, 1000):
        tm = (n + GM - 1) // GM
        ntiles = sum(tm - 2 * c for c in range((tm + 1) // 2))
        covered = {}
        for t in range(ntiles):
            bm, bn = g_tile(t, tm)
            assert 0 <= bm < tm and bm >= 2 * bn
            for i in range(bm * GM, min(n, bm * GM + GM)):
                for j in range(bn * GN, min(i, n - 1, bn * GN + GN - 1) + 1):
                    assert (i, j) not in covered
                    covered[(i, j)] = t
        assert len(covered) == n * (n + 1) // 2


def test_syr2k_k_steps_stay_inside_the_row():
    # the four K16 steps of a chunk advance the descriptor start by 32 bytes:
    # every step reads 32 bytes of each 128-byte row, never across it
    for ks in range(GK // 16):
        assert ks * 32 + 32 <= 128


# ---------------------------------------------------------------------------
# Stage-2 kernel (evd4sc2025_b200/csrc/bc_back.cu): sweep ranges and the
# identity start.  The kernel applies, per column block, strips bottom-up;
# inside a strip the blocks of 8 sweeps of the launch's range in order, inside
# a block the four 32-row groups bottom-up, inside a group the sweeps in order.
# The mixed solve calls it once per chase range, starting from X = I, and a
# CTA skips strip R when R > (first column) + (columns) + 64.

import numpy as np

from oracle import algos as O


def _random_chase_u(n, seed):
    rng = np.random.default_rng(seed)
    U = np.zeros((n, n))
    for s in range(n - 2):
        for r in range(s + 1, n - 1, 32):  # the chase stores no one-row reflector
            seg = rng.standard_normal(min(32, n - r))
            U[r:r + len(seg), s] = seg * np.sqrt(2.0) / np.linalg.norm(seg)
    return U


def _kernel_order(X, U, n, ranges, cols, ident, ident_k=0):
    X = X.copy()
    nstrips = (n - 2 + 127) // 128
    for h0, h1 in ranges:
        for cb in range(0, n, cols):
            cs = slice(cb, min(n, cb + cols))
            for sidx in range(nstrips - 1, -1, -1):
                R = 128 * sidx
                H = n - 2 - R
                nblk = (H + 7) // 8
                bbA, bbB = h0 // 8, min(nblk, (h1 + 7) // 8)
                if bbB <= bbA or (ident and R > cb + cols + 64 - ident_k):
                    continue
                for bb in range(bbA, bbB):
                    for J in range(3, -1, -1):
                        for p in range(8):
                            h = 8 * bb + p
                            if h >= H:
                                continue
                            r0 = R + h + 1 + 32 * J
                            if r0 >= n:
                                continue
                            u = U[r0:r0 + 32, h]
                            X[r0:r0 + 32, cs] -= np.outer(u, u @ X[r0:r0 + 32, cs])
    return X


def test_stage2_ranges_keep_the_generation_order():
    n = 300
    U = _random_chase_u(n, 5)
    X0 = np.random.default_rng(6).standard_normal((n, 40))
    ref = O.q2_apply(X0, U, n, 32, transpose=True)
    for ranges in ([(0, n)], [(0, 64), (64, 200), (200, n - 2)], [(0, 8), (8, n - 2)]):
        got = _kernel_order(X0, U, n, ranges, 40, False)
        assert np.abs(got - ref).max() < 1e-12


def test_stage2_identity_start_support_and_skip():
    n = 420
    U = _random_chase_u(n, 7)
    X = np.eye(n)
    # before sweep h, column c is zero below row c + 30 + h
    for h in range(n - 2):
        rows = np.arange(n)[:, None]
        cols = np.arange(n)[None, :]
        assert np.all(X[rows > cols + 30 + h] == 0.0), h
        for r in range(h + 1, n, 32):
            u = U[r:r + 32, h]
            X[r:r + 32] -= np.outer(u, u @ X[r:r + 32])
    ref = O.q2_apply(np.eye(n), U, n, 32, transpose=True)
    assert np.abs(X - ref).max() < 1e-12
    bounds = [0, 64, 192, n - 2]
    for cols in (32, 64):
        got = _kernel_order(np.eye(n), U, n, list(zip(bounds[:-1], bounds[1:])), cols, True)
        assert np.abs(got - ref).max() < 1e-12


def test_stage2_two_chains_from_the_identity():
    # Q2^T = B A with A = the sweeps [0, k) and B = the sweeps [k, n-2), each
    # applied to the identity (B skips by the shifted rule)
    n, k = 420, 136
    U = _random_chase_u(n, 9)
    ref = O.q2_apply(np.eye(n), U, n, 32, transpose=True)
    for cols in (32, 64):
        A = _kernel_order(np.eye(n), U, n, [(0, 64), (64, k)], cols, True, 0)
        B = _kernel_order(np.eye(n), U, n, [(k, 264), (264, n - 2)], cols, True, k)
        assert np.abs(B @ A - ref).max() < 1e-12
        # B is the identity in its first k + 1 rows and columns
        assert np.array_equal(B[:k + 1, :k + 1], np.eye(k + 1))
        assert not B[:k + 1, k + 1:].any() and not B[k + 1:, :k + 1].any()


# ---------------------------------------------------------------------------
# Panel QR tile factorisation (evd4sc2025_b200/csrc/panel_qr.cu, tile_factor):
# warp w owns columns w, w + 8, ...; the owner of column j + 1 publishes
# reflector j + 1 with bar.arrive on barrier 1 + ((j + 1) & 3), every other
# warp waits on barrier 1 + (j & 3) before applying reflector j.  A barrier
# instance completes once all 8 warps have arrived (arrive or sync).

def _qr_barrier_program(w, nw=8, nb=32):
    ops = [("arrive", 0)] if w == 0 else []
    for j in range(nb):
        if w != (j & 7):
            ops.append(("sync", j))
        if j + 1 < nb and w == ((j + 1) & 7):
            ops.append(("arrive", j + 1))
    return ops


def test_panel_qr_barrier_protocol_cannot_deadlock():
    import random
    nw = 8
    progs = [_qr_barrier_program(w) for w in range(nw)]
    # every column's barrier gets exactly one arrival per warp
    for j in range(32):
        assert sorted(w for w in range(nw) for op in progs[w] if op[1] == j) == list(range(nw))
    rng = random.Random(3)
    for _ in range(3000):
        pc, arrived, current, waiting = [0] * nw, {}, {}, [None] * nw
        while True:
            for w in range(nw):
                if waiting[w] is not None and len(arrived.get(waiting[w], ())) == nw:
                    waiting[w] = None
                    pc[w] += 1
            run = [w for w in range(nw) if pc[w] < len(progs[w]) and waiting[w] is None]
            if not run:
                assert all(pc[w] == len(progs[w]) for w in range(nw)), "deadlock"
                break
            w = rng.choice(run)
            op, j = progs[w][pc[w]]
            bid = 1 + (j & 3)
            open_j = current.get(bid)
            # a barrier id is reused only after its previous instance completed
            assert open_j is None or open_j == j or len(arrived[open_j]) == nw
            current[bid] = j
            arrived.setdefault(j, set()).add(w)
            if op == "arrive":
                pc[w] += 1
            else:
                waiting[w] = j

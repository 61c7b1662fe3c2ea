"""Index arithmetic of the tcgen05 SYR2K kernel, checked on the host (no GPU).

The copy warps of `tc_syr2k_ws_kernel` (evd4sc2025_b200/csrc/lowprec.cu) put
16-byte chunk c (K elements 8c .. 8c+7) of tile row r at
    (r / 8) * 1024 + (r % 8) * 128 + ((c ^ (r % 8)) << 4).
This must (1) stay inside the 16 KB operand tile, (2) give every chunk its
own slot, and (3) equal the 128-byte swizzle the MMA descriptor declares
(SWIZZLE_128B: byte address bits [4:6] XOR bits [7:9] of the row-major
address r * 128 + c * 16).  The global side must read each (row, chunk) of
the packed operand exactly once per stage.
"""

TILE_ROWS, CHUNKS, THREADS = 128, 8, 128


def kernel_offset(row, c):
    return (row >> 3) * 1024 + (row & 7) * 128 + ((c ^ (row & 7)) << 4)


def swizzle128(linear):
    return linear ^ (((linear >> 7) & 7) << 4)


def test_copy_mapping_covers_the_tile_once():
    seen = {}
    for tid in range(THREADS):
        for i in range(TILE_ROWS * CHUNKS // THREADS):
            q = tid + i * THREADS
            row, c = q >> 3, q & 7
            off = kernel_offset(row, c)
            assert off % 16 == 0 and 0 <= off and off + 16 <= TILE_ROWS * 128
            assert off not in seen
            seen[off] = (row, c)
    assert len(seen) == TILE_ROWS * CHUNKS
    assert sorted({rc for rc in seen.values()}) == [(r, c) for r in range(TILE_ROWS)
                                                   for c in range(CHUNKS)]


def test_layout_is_the_128_byte_swizzle():
    for row in range(TILE_ROWS):
        for c in range(CHUNKS):
            assert kernel_offset(row, c) == swizzle128(row * 128 + c * 16)


def test_k_steps_stay_inside_the_row():
    # the four K16 steps of a chunk advance the descriptor start by 32 bytes:
    # every step reads 32 bytes of each 128-byte row, never across it
    for ks in range(4):
        start = ks * 32
        assert start + 32 <= 128


def test_right_operand_rotation_is_chunk_aligned():
    # the right operand [B | A] is row r of H read at K offset (kk + k8) mod L;
    # kk and k8 are multiples of 8, so every 16-byte copy stays inside a row
    for k in (1, 7, 8, 9, 64, 100, 1024):
        k8 = (k + 7) // 8 * 8
        L = 2 * k8
        for kk in range(0, L, 8):
            kr = kk + k8
            if kr >= L:
                kr -= L
            assert kr % 8 == 0 and kr + 8 <= L


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

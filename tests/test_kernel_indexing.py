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

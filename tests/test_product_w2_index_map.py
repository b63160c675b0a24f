"""Host-side check of the width-2 lane-letter product kernel's work map
(roughpy_b200/csrc/product.cu, product_kernel_w2 and launch_levels): a
restatement of its unit, tile and index formulas, checked against the
definitions of a free-tensor product word (level k word w = left word w >> s of
level k - s times right word w mod 2^s of level s) and for exact coverage of
the output levels.  No GPU: this pins the mapping the kernel's comment states."""
import pytest

THREADS = 256
TILE_WORDS = 4096


def units(depth, klo_spec, H):
    """fcum and the unit count per level, as launch_levels builds them."""
    E = H.bit_length() - 1
    low = 6 + E
    klo = max(low, klo_spec)
    fcum, f = {}, 0
    for k in range(klo, depth + 1):
        fcum[k] = f
        f += (1 << (k - 1)) // H
    for k in range(depth + 1, depth + 3):
        fcum[k] = f
    return klo, fcum, f


def walk(depth, klo_spec=1, H=4):
    """Every (level, word, split) the kernel touches, with the indices it uses."""
    E = H.bit_length() - 1
    klo, fcum, ftotal = units(depth, klo_spec, H)
    tile_r = max(THREADS, TILE_WORDS // (2 * H))
    assert tile_r % 32 == 0 and all(v % 32 == 0 for v in fcum.values())
    for bx in range(-(-ftotal // tile_r)):
        f_begin, f_end = bx * tile_r, min(bx * tile_r + tile_r, ftotal)
        for tid in range(THREADS):
            f = f_begin + tid
            while f < f_end:
                k = klo
                while f >= fcum[k + 1]:
                    k += 1
                rp = f - fcum[k]
                lane = tid & 31
                h0 = (rp >> 5) << E
                half = 1 << (k - 1)
                wb = ((1 << k) - 1) + h0 * 32 + lane
                for u in range(2):
                    for i in range(H):
                        o = wb + u * half + 32 * i
                        w = o - ((1 << k) - 1)
                        splits = []
                        for s in range(1, 5):
                            p = k - s
                            r = ((1 << s) - 1) + (lane & ((1 << s) - 1))
                            lb = ((1 << p) - 1) + h0 * (32 >> s) + (lane >> s)
                            splits.append((s, lb + u * (1 << (p - 1)) + (32 >> s) * i, r))
                        for e in range(E):
                            s, nr = 5 + e, 1 << e
                            p = k - s
                            g, c = divmod(i, nr)
                            splits.append((s, ((1 << p) - 1) + (h0 >> e) + u * (1 << (p - 1)) + g,
                                           ((1 << s) - 1) + 32 * c + lane))
                        for s in range(5 + E, k):
                            p = k - s
                            rb = ((1 << s) - 1) + (h0 & ((1 << (s - 5)) - 1)) * 32 + lane
                            lb = ((1 << p) - 1) + (h0 >> (s - 5))
                            splits.append((s, lb + u * (1 << (p - 1)), rb + 32 * i))
                        yield k, w, o, splits
                f += THREADS


@pytest.mark.parametrize("depth,klo_spec,H", [(10, 1, 4), (11, 1, 4), (12, 1, 4), (13, 1, 4),
                                              (12, 10, 4), (12, 12, 4), (12, 1, 8)])
def test_lane_letter_map_covers_and_indexes_exactly(depth, klo_spec, H):
    low = 6 + H.bit_length() - 1
    seen = {}
    for k, w, o, splits in walk(depth, klo_spec, H):
        assert 0 <= w < (1 << k) and o == (1 << k) - 1 + w
        seen[o] = seen.get(o, 0) + 1
        assert [s for s, _, _ in splits] == list(range(1, k))
        for s, li, ri in splits:
            p = k - s
            assert li == (1 << p) - 1 + (w >> s), (k, w, s)           # left word of level p
            assert ri == (1 << s) - 1 + (w & ((1 << s) - 1)), (k, w, s)   # right word of level s
    first = (1 << max(low, klo_spec)) - 1
    assert sorted(seen) == list(range(first, (1 << (depth + 1)) - 1))
    assert set(seen.values()) == {1}


def test_a_warp_shares_level_and_block():
    """The 32 lanes of a warp always hold one level and one block h0, so the
    left-word loads are broadcasts and the right runs coalesce."""
    H = 4
    klo, fcum, ftotal = units(12, 1, H)
    for warp_first in range(0, ftotal, 32):
        ks = set()
        for f in range(warp_first, warp_first + 32):
            k = klo
            while f >= fcum[k + 1]:
                k += 1
            ks.add((k, (f - fcum[k]) >> 5))
        assert len(ks) == 1

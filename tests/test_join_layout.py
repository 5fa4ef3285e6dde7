"""CPU checks of the arithmetic the shared-memory hash join build relies on,
with the library's own sizing helpers (no GPU needed).

The build gives each 16,384-slot region of the table to one block.  A key's
home slot is (hash32(k) * cap) >> 32, so region r owns the hashes
[ceil(r 2^46 / cap), ceil((r + 1) 2^46 / cap)); with
olap_hashjoin_build_filtered the block also sets the Bloom bits of its keys,
whose filter word is hash32(k) >> (32 - log2(words)), so it owns a run of
filter words.  These tests restate that arithmetic (as the kernel
smem_region_build_kernel computes it) and check the three facts the kernel
needs: the hash ranges of the regions tile [0, 2^32) exactly as the home slot
assigns them; a region's run of words fits the kernel's shared buffer
(kSmemFilterWords = 2064) for every size the helpers produce, so the fused
path is always the one taken; and only a run's first and last words can be
shared with a neighbouring region (those the kernel ORs into the filter)."""

import numpy as np
import pytest

from memory_database_b200 import _lib

REGION_SHIFT = 14      # 16,384 slots a region
FILTER_WORDS = 2064    # the build kernel's shared filter buffer, in words
MAX_SLOTS = 1 << 27    # largest table built in shared memory


def region_hashes(r, cap):
    """[h_lo, h_hi) of region r, as the kernel computes them (h_hi clamped)."""
    h_lo = ((r << (32 + REGION_SHIFT)) + cap - 1) // cap
    h_hi = (((r + 1) << (32 + REGION_SHIFT)) + cap - 1) // cap
    return h_lo, min(h_hi, 1 << 32)


def home(h, cap):
    return (h * cap) >> 32


def sizes():
    """(build rows, capacity, filter words) as a caller of the helpers gets
    them, for the tables the shared-memory build takes (above 2^22 slots)."""
    lib = _lib.lib
    rng = np.random.default_rng(5)
    ns = [(1 << 21) + 1, (1 << 21) + 12_345, 3_000_000, 1 << 24, (1 << 24) + 7, 40_000_000,
          (1 << 26) - 1, (1 << 26) - 5]
    ns += [int(x) for x in rng.integers((1 << 21) + 1, 1 << 26, 24)]
    out = []
    for n in ns:
        cap = int(lib.olap_hashtable_capacity(n))
        if (1 << 22) < cap <= MAX_SLOTS:
            out.append((n, cap, int(lib.olap_hashjoin_filter_words(n))))
    assert len(out) > 20
    return out


@pytest.mark.parametrize("n,cap,words", sizes())
def test_regions_tile_the_hash_space(n, cap, words):
    P = (cap + (1 << REGION_SHIFT) - 1) >> REGION_SHIFT
    for r in sorted({0, 1, P // 3, P // 2, P - 2, P - 1}):
        h_lo, h_hi = region_hashes(r, cap)
        assert home(h_lo, cap) >> REGION_SHIFT == r
        assert home(h_hi - 1, cap) >> REGION_SHIFT == r
        if r:
            assert home(h_lo - 1, cap) >> REGION_SHIFT == r - 1
    assert region_hashes(0, cap)[0] == 0 and region_hashes(P - 1, cap)[1] == 1 << 32


@pytest.mark.parametrize("n,cap,words", sizes())
def test_filter_runs_fit_and_share_only_their_ends(n, cap, words):
    lg = words.bit_length() - 1
    assert 1 << lg == words
    fshift = 32 - lg
    P = (cap + (1 << REGION_SHIFT) - 1) >> REGION_SHIFT
    # the host's test for the fused path
    per_region = ((1 << (32 + REGION_SHIFT)) + cap - 1) // cap
    assert (per_region >> fshift) + 2 <= FILTER_WORDS
    prev_hi_word = -1
    for r in range(P):
        h_lo, h_hi = region_hashes(r, cap)
        w_lo, w_hi = h_lo >> fshift, (h_hi - 1) >> fshift
        assert w_hi - w_lo + 1 <= FILTER_WORDS
        # the words strictly inside the run hold only this region's hashes
        if w_hi - w_lo >= 2:
            assert (w_lo + 1) << fshift >= h_lo and w_hi << fshift <= h_hi
        # consecutive runs meet or touch at their end words only
        assert w_lo in (prev_hi_word, prev_hi_word + 1) or r == 0
        prev_hi_word = w_hi
    assert prev_hi_word == words - 1

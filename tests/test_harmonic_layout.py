"""CPU model of the harmonic kernel's memory accesses (csrc/harmonic_fast.cu).

The kernel's index arithmetic is restated here and checked exhaustively, so
that its bulk staging copies and its direct vector loads are known to stay
inside the power spectrum and the shared staging buffer, and to be aligned as
cp.async.bulk and 8/16-byte loads require:

* CTA x owns the 16-bin blocks m' = 127 x .. 127 x + 126 (thread m = 1..127;
  thread 0 computes the halo of block 127 x - 1), so the grid covers every
  block below the largest span;
* odd factor k is staged as region_floats(k) floats from the 16-byte aligned
  ga = floor4(first k); thread m reads region[m k + o + (first k - ga)],
  o < NV(k) = ((15 k + 8) >> 4) + 1, and those are exactly P[(first + m) k + o];
* an interior CTA (first >= 0 and floor4(15 first) + region_floats(15) <= M)
  stages every odd factor with one bulk copy inside [0, M);
* a thread whose block is inside [0, M) ("direct") reads its even factors and
  the level-0 values with 8-byte (k = 2 mod 4) or 16-byte (k = 0 mod 4) vector
  loads that are aligned and end below (m' + 1) 16 <= M.
"""
import numpy as np
import pytest

THREADS = 128
BLOCKS = THREADS - 1


def region_floats(k):
    return ((THREADS * k + 1 + 3 + 3) // 4) * 4


def odd_base(k):
    return sum(region_floats(q) for q in range(1, k, 2))


def nv(k):
    return ((15 * k + 8) >> 4) + 1


def floor4(x):
    return x & ~3 if x >= 0 else -((-x + 3) & ~3)


def test_staging_regions_aligned_and_fit_six_ctas_per_sm():
    stage = odd_base(17)
    for k in range(1, 17, 2):
        assert region_floats(k) % 4 == 0 and odd_base(k) % 4 == 0  # 16-byte copies, 16-byte destinations
    assert stage * 4 <= 33 * 1024
    assert 6 * (stage * 4 + 1024 + 256) <= 228 * 1024  # + reserved and static shared memory per CTA


@pytest.mark.parametrize("k", list(range(1, 17, 2)))
def test_odd_factor_reads_stay_in_their_region(k):
    for first in list(range(-1, 64)) + [127 * 1000 - 1, 127 * 16513 - 1]:
        ga = floor4(first * k)
        d = first * k - ga
        assert 0 <= d <= 3
        m = np.arange(THREADS)
        o = np.arange(nv(k))[:, None]
        e = m * k + o + d  # region element
        assert e.min() >= 0 and e.max() < region_floats(k)
        assert np.array_equal(ga + e, (first + m) * k + o)  # the power values the thread needs


def test_interior_ctas_stage_inside_the_spectrum():
    for M in (1 << 12, 3 << 13, 1 << 19, 3 << 20, 1 << 21, 3 << 21):
        last = (M // 16 + BLOCKS - 1) // BLOCKS + 2
        for x in range(last):
            first = x * BLOCKS - 1
            bulk = first >= 0 and floor4(first * 15) + region_floats(15) <= M
            if not bulk:
                continue
            for k in range(1, 17, 2):
                ga = floor4(first * k)
                assert ga >= 0 and ga + region_floats(k) <= M, (M, x, k)


def test_grid_covers_every_block():
    for span in (1, 16, 17, 2032, 2033, 2049, (1 << 21) + 8, 3 << 20):
        blocks16 = (span + 15) // 16
        ctas = max((blocks16 + BLOCKS - 1) // BLOCKS, 1)
        owned = {x * BLOCKS - 1 + m for x in range(ctas) for m in range(1, THREADS)}
        assert set(range(blocks16)) <= owned


@pytest.mark.parametrize("k", [2, 4, 6, 8, 10, 12, 14, 16])
def test_direct_vector_loads_aligned_and_in_bounds(k):
    width = 4 if k % 4 == 0 else 2  # floats per vector load
    loads = (nv(k) + width - 1) // width
    for mp in range(0, 4096):
        start = mp * k
        assert (start * 4) % (4 * width) == 0  # 16- or 8-byte aligned: each spectrum starts 16-byte aligned (M floats apart, M >= 4096)
        end = start + loads * width  # one past the last float read
        assert end <= (mp + 1) * 16  # inside the thread's own bound: direct means (m' + 1) 16 <= M
        assert loads * width >= nv(k)


def test_direct_load_line_counts():
    """Lines of 128 bytes a warp's direct loads touch (32 consecutive blocks):
    a vector load of factor k spans 32 windows k floats apart, so the even
    factors and the level-0 values touch 312 lines per warp for 72 lines of
    data; the odd factors' staged reads are 68 conflict-free shared accesses."""
    touched = data = 0
    for k in (2, 4, 6, 8, 10, 12, 14, 16):
        width = 4 if k % 4 == 0 else 2
        for v in range((nv(k) + width - 1) // width):
            lines = set()
            for lane in range(32):
                a = ((32000 + lane) * k + v * width) * 4
                lines.update(range(a // 128, (a + 4 * width - 1) // 128 + 1))
            touched += len(lines)
        data += (32 * k * 4) // 128
    assert (touched, data) == (312, 72)
    assert sum(nv(k) for k in range(1, 17, 2)) == 68

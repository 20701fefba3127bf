"""CPU model of pass 2's power-spectrum writes (csrc/fused_fast.cu `pass2_fast`).

Pass 2 CTA q holds rows qR .. qR + R - 1 of the four-step intermediate and their
mirrors L1 - (qR + r) (row L1/2 in place of row 0's mirror), so that each CTA
has both Z_k and Z_{M-k} of its bins.  CTAs q > 0 write the bin pair
k = arow + L1 k2, km = brow + L1 (L2 - 1 - k2) from thread (r, j) and its
butterfly outputs m (k2 = j + Ns m, `pass2_pairs`); CTA 0 walks k2 = t / R +
it THREADS / R, writing the pairs of rows 1 .. R - 1 and the self-paired rows
0 (bins L1 k2, with P[0] = 0) and L1/2 (bins L1/2 + L1 k2).  The model checks,
for every compiled pass-2 configuration and the row counts L1 it pairs with,
that the CTAs' writes cover the spectrum [0, M) exactly once.
"""
import numpy as np
import pytest

# id: (L2, R row pairs, THREADS, radix of the last pass)
PASS2 = {201: (1024, 2, 256, 8), 202: (1024, 4, 512, 8), 203: (512, 4, 256, 8), 204: (2048, 2, 512, 8),
         205: (512, 8, 512, 8), 207: (2048, 4, 1024, 8)}
L1S = (512, 1024, 1536, 2048, 3072)
FIRST_RADIX = {201: 16, 202: 16, 203: 8, 204: 16, 205: 8, 207: 16}  # first pass of each radix sequence


def written_bins(L1, L2, R, THREADS, RL):
    M = L1 * L2
    Ns = L2 // RL
    assert R * Ns == THREADS, "one bin-pair butterfly pair per thread"
    out = []
    # CTAs q > 0: pass2_pairs
    q = np.arange(1, L1 // (2 * R))[:, None, None, None]
    t = np.arange(THREADS)[None, :, None, None]
    r, j = t % R, t // R
    m = np.arange(RL)[None, None, :, None]
    k2 = j + Ns * m
    arow = q * R + r
    brow = L1 - arow
    out.append((arow + L1 * k2).ravel())
    out.append((brow + L1 * (L2 - 1 - k2)).ravel())
    # CTA 0: rows 0 .. R - 1 with their mirrors; row 0 with itself and row L1/2 with itself
    KSTEP, ITER = THREADS // R, R * L2 // THREADS
    t = np.arange(THREADS)
    for it in range(ITER):
        k2 = t // R + it * KSTEP
        r = t % R
        zero = r == 0
        out.append(L1 * k2[zero])
        out.append(L1 // 2 + L1 * k2[zero])
        a = r[~zero]
        kk2 = k2[~zero]
        out.append(a + L1 * kk2)
        out.append((L1 - a) + L1 * (L2 - 1 - kk2))
    return M, np.concatenate(out)


@pytest.mark.parametrize("cfg", sorted(PASS2))
@pytest.mark.parametrize("L1", L1S)
def test_power_bins_written_exactly_once(cfg, L1):
    L2, R, THREADS, RL = PASS2[cfg]
    if L1 % (2 * R):
        pytest.skip("the plan pairs this pass 2 only with L1 divisible by 2R")
    M, bins = written_bins(L1, L2, R, THREADS, RL)
    assert bins.min() == 0 and bins.max() == M - 1
    counts = np.bincount(bins, minlength=M)
    assert np.all(counts == 1), (np.flatnonzero(counts != 1)[:8], M)


def pass2_row(rr, R, q, L1):
    """Row of sequence rr of CTA q (fused_fast.cu pass2_row)."""
    if rr < R:
        return q * R + rr
    ar = q * R + (rr - R)
    return L1 // 2 if ar == 0 else L1 - ar


@pytest.mark.parametrize("R", [2, 4, 8])
@pytest.mark.parametrize("L1", L1S)
def test_every_row_loaded_by_exactly_one_cta(R, L1):
    """The CTAs' 2R rows (R rows and their mirrors) partition the L1 rows of
    the intermediate; CTA 0 holds the self-paired rows 0 and L1/2."""
    if L1 % (2 * R):
        pytest.skip("the plan pairs R row pairs only with L1 divisible by 2R")
    rows = [pass2_row(rr, R, q, L1) for q in range(L1 // (2 * R)) for rr in range(2 * R)]
    assert sorted(rows) == list(range(L1))
    assert {pass2_row(0, R, 0, L1), pass2_row(R, R, 0, L1)} == {0, L1 // 2}
    for q in range(1, L1 // (2 * R)):  # a mirror row pairs Z_k with Z_{M-k}: row a with row L1 - a
        for r in range(R):
            assert pass2_row(r, R, q, L1) + pass2_row(R + r, R, q, L1) == L1


@pytest.mark.parametrize("cfg", sorted(PASS2))
def test_first_pass_row_loads_cover_the_rows(cfg):
    """With the first radix-16 pass on the loads (2R L2 = 16 THREADS), thread
    t loads inputs j + r L2/16 (r < 16) of sequence t / (L2/16), j = t % (L2/16):
    every element of the CTA's 2R rows once."""
    L2, R, THREADS, _ = PASS2[cfg]
    if 2 * R * L2 != 16 * THREADS or FIRST_RADIX[cfg] != 16:
        pytest.skip("this configuration loads its rows in shared memory first")
    nbf = L2 // 16
    t = np.arange(THREADS)[:, None]
    r = np.arange(16)[None, :]
    elem = (t // nbf) * L2 + (t % nbf) + r * nbf
    assert np.array_equal(np.sort(elem.ravel()), np.arange(2 * R * L2))

"""CPU model of the warp-local pass 1 (csrc/pass1_warp.cu, configurations
124-127): which complex points each thread gathers, and its shared-memory
exchange.

* The CTAs of a template gather every complex point p = L2 (j + r L1/16) + c0 + c
  of the M = L1 L2 packed series exactly once (thread (w, lane): column
  c = lane % C, first-pass butterfly j = w + 16 (lane / C), inputs r = 0..15).
* Middle pass without a block barrier: in warp w's region of column c, lane
  q = lane / C reads and then writes exactly the slots (r, MB q .. MB q + MB - 1),
  r < R2, of the R2 x 16 first-pass outputs; these sets are disjoint across the
  lanes and cover the region's 16 R2 outputs, so no lane's write can meet
  another lane's read (hence __syncwarp alone).
* The last pass (after the block barrier) reads every first-pass/middle slot of
  every region exactly once.
* Bank model (32 banks of 4 bytes; a warp's 16-byte accesses in quarter warps,
  8-byte ones in half warps; a word read by several lanes is one access): the
  first-pass row stores, the middle pass's loads and stores, the last pass's
  loads and the column-factor table are free of bank conflicts.
"""
import numpy as np
import pytest

ROW_STRIDE = 18
SHAPES = [(8, 4), (4, 8)]  # (R2, C): configurations 124/126 and 125/127


def layout(R2, C):
    shift = 16 // C
    reg = R2 * ROW_STRIDE + (shift - R2 * ROW_STRIDE) % 16
    return reg, (lambda w, c: (w * C + c) * reg)


def wavefronts(addrs, width):
    """Shared-memory wavefronts of one warp access (byte addresses per lane)."""
    per = {16: 8, 8: 16, 4: 32}[width]
    total = 0
    for p0 in range(0, len(addrs), per):
        banks = {}
        for a in addrs[p0:p0 + per]:
            for k in range(width // 4):
                word = a // 4 + k
                banks.setdefault(word % 32, set()).add(word)
        total += max(len(v) for v in banks.values())
    return total


@pytest.mark.parametrize("R2,C", SHAPES)
@pytest.mark.parametrize("L2", [512, 1024, 2048])
def test_gather_covers_every_complex_point_once(R2, C, L2):
    L1 = 256 * R2
    NBF = L1 // 16
    lane = np.arange(32)
    c, q = lane % C, lane // C
    w = np.arange(16)[:, None, None]
    j = w + 16 * q[None, :, None]
    r = np.arange(16)[None, None, :]
    cols = (c[None, :, None] + 0 * r)
    seen = np.zeros(L1 * L2, np.int32)
    for c0 in range(0, L2, C):
        p = L2 * (j + r * NBF) + c0 + cols
        np.add.at(seen, p.ravel(), 1)
    assert np.all(seen == 1)


@pytest.mark.parametrize("R2,C", SHAPES)
def test_middle_pass_ownership_needs_no_barrier(R2, C):
    MB = 16 // R2
    owned = {}
    for qq in range(R2):  # lane q of a column: reads and writes the same slots
        slots = {(r, MB * qq + u) for r in range(R2) for u in range(MB)}
        for s in slots:
            assert s not in owned
            owned[s] = qq
    assert set(owned) == {(r, m) for r in range(R2) for m in range(16)}


@pytest.mark.parametrize("R2,C", SHAPES)
def test_last_pass_reads_every_slot_once(R2, C):
    reg, base = layout(R2, C)
    seen = {}
    for t in range(512):
        cc, jp = t % C, t // C
        for r in range(16):
            a = base(r, cc) + ROW_STRIDE * (jp // 16) + jp % 16
            seen[a] = seen.get(a, 0) + 1
    expect = {base(w, c) + ROW_STRIDE * rr + m for w in range(16) for c in range(C) for rr in range(R2)
              for m in range(16)}
    assert set(seen) == expect and all(v == 1 for v in seen.values())
    assert max(expect) < 16 * C * reg  # inside the exchange buffer


@pytest.mark.parametrize("R2,C", SHAPES)
def test_exchange_is_free_of_bank_conflicts(R2, C):
    reg, base = layout(R2, C)
    MB = 16 // R2
    lane = np.arange(32)
    c, q = lane % C, lane // C
    for w in range(16):
        for h in range(8):  # first-pass outputs: 8 float4 per lane
            a = [8 * (base(w, cc) + ROW_STRIDE * qq + 2 * h) for cc, qq in zip(c, q)]
            assert wavefronts(a, 16) == 4
        for r in range(R2):  # middle pass: MB/2 float4 per row, loaded then stored
            for h in range(MB // 2):
                a = [8 * (base(w, cc) + ROW_STRIDE * r + MB * qq + 2 * h) for cc, qq in zip(c, q)]
                assert wavefronts(a, 16) == 4
        t = np.arange(32 * w, 32 * w + 32)
        cc, jp = t % C, t // C
        for r in range(16):  # last pass: one float2 from every warp's region
            a = [8 * (base(r, x) + ROW_STRIDE * (j // 16) + j % 16) for x, j in zip(cc, jp)]
            assert wavefronts(a, 8) == 2
        for m in range(16):  # column factors s_fs[C][17]
            assert wavefronts([8 * (x * 17 + m) for x in cc], 8) <= 2

"""CPU model of the bulk tensor store of pass 1 (configurations 126 and 127,
csrc/pass1_warp.cu `pass1_warp_tma`; 128, csrc/fused_fast.cu `pass1_fast_tma`).

The kernel's index arithmetic is restated here and checked exhaustively for
both compiled shapes, so that every shared-memory write and every bulk copy the
kernel issues is known to stay inside its buffers and to meet the alignment
rules of cp.async.bulk.tensor before it runs on a device:

* thread t = C jp + cc writes its 16 outputs m to tile[(jp + m L1/16) C + cc]:
  every (row, column) of the L1 x C tile exactly once, a warp's 32 stores of
  one m 256 contiguous bytes;
* the tile starts at the first 128-byte boundary of the exchange buffer and
  ends inside it, whatever the buffer's own alignment (at least 16 bytes);
* box b (256 rows) starts 256 b C 8 bytes into the tile, so every box source
  is 128-byte aligned and the L1/256 boxes cover the tile once;
* the innermost box coordinate c0 = C blockIdx.x times 8 bytes is a multiple
  of 16 for every CTA, the box's inner extent C 8 bytes is one too, the box
  rows 256 b .. 256 b + 255 lie inside the L1 rows and the columns inside L2;
* the tensor map's strides (L2 8 and M 8 bytes) are multiples of 16.
"""
import numpy as np
import pytest

ROW_STRIDE = 18  # float2 per row of 16 values in a warp region (kRowStride)
THREADS = 512
SHAPES = [(8, 4, 126), (4, 8, 127)]  # (R2, C, config id)


def warp_layout(r2, c):
    """WarpLayout<R2, C>: region size REG and the exchange buffer in bytes."""
    shift = 16 // c
    reg = r2 * ROW_STRIDE + (shift - r2 * ROW_STRIDE) % 16  # C++ ((x % 16) + 16) % 16 == Python x % 16
    assert reg % 16 == shift % 16 and reg >= r2 * ROW_STRIDE and reg % 2 == 0
    return reg, 16 * c * reg * 8


@pytest.mark.parametrize("r2,c,cfg", SHAPES)
def test_tile_writes_cover_the_tile_once_and_coalesce(r2, c, cfg):
    l1 = 256 * r2
    nbf = l1 // 16
    t = np.arange(THREADS)
    cc, jp = t % c, t // c
    m = np.arange(16)[:, None]
    idx = (jp[None, :] + m * nbf) * c + cc[None, :]  # [m][thread]
    assert idx.min() == 0 and idx.max() == l1 * c - 1
    assert np.array_equal(np.sort(idx.ravel()), np.arange(l1 * c))
    # one warp, one m: 32 consecutive float2 starting on a 256-byte boundary
    w = idx.reshape(16, THREADS // 32, 32)
    assert np.all(np.diff(w, axis=2) == 1)
    assert np.all((w[:, :, 0] * 8) % 256 == 0)
    # row and column of each write are the butterfly's output row and column
    assert np.array_equal(idx // c, jp[None, :] + m * nbf)
    assert np.array_equal(idx % c, np.broadcast_to(cc, idx.shape))


@pytest.mark.parametrize("r2,c,cfg", SHAPES)
def test_tile_and_boxes_fit_the_exchange_buffer(r2, c, cfg):
    l1 = 256 * r2
    _, smem = warp_layout(r2, c)
    tile = l1 * c * 8
    assert tile == 65536
    for base in range(0, 4096, 16):  # every 16-byte aligned start of the dynamic buffer
        tile_sh = (base + 127) & ~127
        assert tile_sh - base <= 112 and (tile_sh - base) % 8 == 0  # a whole number of float2
        assert tile_sh + tile <= base + smem
        boxes = [tile_sh + b * 256 * c * 8 for b in range(l1 // 256)]
        assert all(s % 128 == 0 for s in boxes)
        assert boxes[-1] + 256 * c * 8 == tile_sh + tile  # boxes tile the tile, none past it
    assert l1 // 256 == r2


@pytest.mark.parametrize("r2,c,cfg", SHAPES)
@pytest.mark.parametrize("l2", [512, 1024, 2048])
def test_box_coordinates_meet_the_tma_rules(r2, c, cfg, l2):
    l1 = 256 * r2
    m_len = l1 * l2
    assert (c * 8) % 16 == 0 and c <= 256  # inner box extent
    assert (l2 * 8) % 16 == 0 and (m_len * 8) % 16 == 0  # global strides
    c0 = np.arange(l2 // c) * c  # blocks = L2 / C CTAs per template
    assert np.all((c0 * 8) % 16 == 0)  # innermost coordinate x element size
    assert np.all(c0 >= 0) and np.all(c0 + c <= l2)
    ys = 256 * np.arange(l1 // 256)
    assert np.all(ys >= 0) and np.all(ys + 256 <= l1)


def ct_stride(L, G):
    """Exchange-buffer stride of pass1_fast (fast_common.cuh ct_stride)."""
    base = L + L // 16
    want = 1 if G >= 16 else 16 // G
    return base + (want - base) % 16


def test_pass1_fast_tile_config_128():
    """Config 128 = 119 (L1 = 1536 = 16.4.3.8, 4 columns, 384 threads) with the
    bulk store: the last radix-8 pass (span 192) of ct_last_pass_tile writes
    thread t's outputs of butterflies j = t/4 + 96 q (q = 0, 1) to
    tile[(j + 192 m) 4 + t % 4]."""
    L1, C, THREADS, R = 1536, 4, 384, 8
    Ns = NBF = L1 // R
    PER = NBF * C // THREADS
    assert PER * THREADS == NBF * C and Ns * R == L1
    t = np.arange(THREADS)
    c = t % C
    idx = np.stack([(t // C + q * (THREADS // C) + m * Ns) * C + c for q in range(PER) for m in range(R)])
    assert np.array_equal(np.sort(idx.ravel()), np.arange(L1 * C))
    w = idx.reshape(PER * R, THREADS // 32, 32)
    assert np.all(np.diff(w, axis=2) == 1) and np.all((w[:, :, 0] * 8) % 256 == 0)
    smem = C * ct_stride(L1, C) * 8
    assert smem >= L1 * C * 8 + 128 and L1 % 256 == 0
    for base in range(0, 4096, 16):
        tile_sh = (base + 127) & ~127
        assert tile_sh + L1 * C * 8 <= base + smem and (tile_sh - base) % 8 == 0
    for l2 in (512, 1024, 2048):  # the pass-2 row lengths it pairs with
        c0 = np.arange(l2 // C) * C
        assert np.all((c0 * 8) % 16 == 0) and np.all(c0 + C <= l2)


def test_compiled_bulk_store_configs_are_listed():
    from brp_b200._lib import fast_configs
    cfg = {i: (L, k) for i, L, k in fast_configs()}
    for r2, c, cid in SHAPES:
        assert cfg[cid] == (256 * r2, 1)  # pass 1, L1 = 256 R2
    assert cfg[124] == (2048, 1) and cfg[125] == (1024, 1)  # the plain-store forms stay compiled
    assert cfg[128] == (1536, 1) and cfg[119] == (1536, 1)

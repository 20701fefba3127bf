"""The C-ABI library loads without a GPU and exports every function that
include/brp_cuda.h declares; the oracle library exports its C interface."""
import ctypes
import os
import re

import brp_b200 as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(brp_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    names = declared(os.path.join(ROOT, "include", "brp_cuda.h"))
    assert len(names) >= 25
    lib = ctypes.CDLL(B.build())
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(B.EXPORTS) <= set(names)


def test_params_layout_matches_reference():
    assert ctypes.sizeof(B.Params) == 108
    assert B.Params.threshold.offset == 56 and B.Params.result_slot.offset == 104
    assert B.CANDIDATE.itemsize == 16 and B.BANK_CANDIDATE.itemsize == 48


def test_errors_without_device_are_reported():
    # no CUDA device here: creating a context fails with a message, never crashes
    import numpy as np
    import pytest
    p = B.parameters(8192, 8000, 0.1, 600.0, 0.0, 128e-6)
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(B.BrpError) as e:
        B.GPU(p, np.zeros(8000, np.float32), 192, 0, 1)
    assert str(e.value)


def test_option_validation_matches_reference():
    # src/vulkan.cpp:278-284: flag combinations are rejected before any device work
    import numpy as np
    import pytest
    p = B.parameters(8192, 8000, 0.1, 600.0, 0.0, 128e-6)
    x = np.zeros(8000, np.float32)
    for kw in (dict(fused_power=True), dict(radix8_store=True), dict(radix8=True, stockham=False),
               dict(stockham=True, tile=512)):
        args = dict(workgroup=192, tile=0, batch=1)
        args.update(kw)
        with pytest.raises(B.BrpError) as e:
            B.GPU(p, x, **args)
        assert e.value.status == 1


def test_oracle_library_exports():
    from oracle import oracle as O
    L = O.lib()
    for name in ("oracle_resample", "oracle_harmonic", "oracle_select", "oracle_search_parameters",
                 "oracle_toplist_retain", "oracle_toplist_final", "oracle_rfft64"):
        assert hasattr(L, name)


def test_tensor_core_pass1_configs_listed():
    """The tensor-core pass-1 forms (kind 3) sit beside the CUDA-core pass-1
    configuration of the same column length and never enter the autotuner."""
    from brp_b200 import tune
    from brp_b200._lib import fast_configs
    kinds = {i: (L, k) for i, L, k in fast_configs()}
    for tc, base in ((111, 110), (112, 110), (113, 119), (114, 119)):
        assert kinds[tc] == (kinds[base][0], 3)
    ids = {c[0] for c in tune.candidates(1 << 22) + tune.candidates(3 << 21)}
    assert ids and not ids & {111, 112, 113, 114}


def test_argument_errors_of_the_whitening_and_filter_entry_points():
    """Invalid arguments are rejected before any device work (no GPU needed):
    a series longer than n, an unsupported length, a packed DD series of odd
    length, a missing bank."""
    import ctypes

    import numpy as np
    import pytest
    from brp_b200 import whiten
    from brp_b200._lib import lib
    x = np.zeros(10000, np.float32)
    with pytest.raises(B.BrpError, match="invalid observation"):
        whiten.preprocess(x, 8192, 128.0, 1.0, 1000)
    with pytest.raises(B.BrpError, match="2\\^k or 3\\*2\\^k"):
        whiten.preprocess(x, 10000, 128.0, 1.0, 1000)
    with pytest.raises(B.BrpError, match="invalid DD metadata"):
        whiten.preprocess_dd(np.zeros(5000, np.uint8), 9999, True, 2.0, 16384, 128.0, 1.0, 1000)
    L = lib()
    assert L.brp_cuda_bank_set_toplist_filter(ctypes.c_void_p(0), 100) == 4


def test_static_search_rejects_misaligned_buffers():
    """brp_cuda_search_static checks the alignment its kernels need (16 bytes
    for the power spectrum and the candidates, 4 for the rest) before any
    device work, so a misaligned view is an argument error, not a fault."""
    import ctypes
    from brp_b200._lib import as_params, lib
    p = as_params(B.parameters(1 << 16, (1 << 16) - 17, 0.3, 3600.0, 1.1, 128e-6))
    L = lib()
    ok, word = 1 << 12, 1 << 12  # aligned stand-in addresses (never dereferenced)
    cases = [(ok, ok + 4, ok, word, word), (ok, ok, ok + 8, word, word), (ok + 2, ok, ok, word, word),
             (ok, ok, ok, word + 1, word), (ok, ok, ok, word, word + 2)]
    for inp, power, cands, count, status in cases:
        st = L.brp_cuda_search_static(ctypes.byref(p), ctypes.c_void_p(inp), ctypes.c_void_p(power),
                                      ctypes.c_void_p(cands), 16, ctypes.c_void_p(count), ctypes.c_void_p(status),
                                      None)
        assert st == 4
        assert b"aligned" in L.brp_cuda_search_static_error()


def test_wait_limit_entry_points_check_their_arguments():
    import ctypes
    from brp_b200._lib import lib
    L = lib()
    assert L.brp_cuda_set_wait_limits(ctypes.c_void_p(0), 10, 1.0) == 4
    assert L.brp_cuda_bank_set_wait_limits(ctypes.c_void_p(0), 10, 1.0) == 4
    L.brp_cuda_debug_fail_allocation(0)  # off: a no-op without a device


def test_plan_file_is_read_without_a_device(tmp_path):
    """The plan file shared with the Python tuner (json.dump of
    {key: {pass1, pass2, group, chains, ms}}) is accepted; a malformed one or a
    missing one is an argument error; "" resets to the built-in plans."""
    import json
    from brp_b200._lib import lib
    L = lib()
    good = tmp_path / "plans.json"
    json.dump({"B200/sm100/148|n=4194304|templates=512": {"chains": 1, "group": 128, "ms": 15.4, "pass1": 110,
                                                          "pass2": 202},
               "B200/sm100/148|n=6291456|templates=128": {"pass1": 119, "pass2": 204, "group": 128, "chains": 2,
                                                          "ms": 7.5, "tried": [1, 2, {"x": None}]}},
              open(good, "w"), indent=1, sort_keys=True)
    assert L.brp_cuda_load_plan_cache(str(good).encode()) == 0
    bad = tmp_path / "bad.json"
    bad.write_text('{"k": {"pass1": 1, "pass2": }')
    assert L.brp_cuda_load_plan_cache(str(bad).encode()) == 4
    assert b"invalid plan cache" in L.brp_cuda_autotune_error()
    assert L.brp_cuda_load_plan_cache(str(tmp_path / "missing.json").encode()) == 4
    assert L.brp_cuda_load_plan_cache(b"") == 0

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

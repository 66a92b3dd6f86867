"""CPU-side checks of the C-ABI library: it loads, exports every function that
include/minipoa_b200.h declares, and fails loudly without a CUDA device."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "minipoa_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(poa_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for required in ["poa_align_sequences", "poa_extend_graph", "poa_align", "poa_poa", "poa_graph_add_path",
                     "poa_graph_toposort", "poa_graph_consensus", "poa_graph_msa", "poa_graph_gfa",
                     "poa_dp_backend", "poa_batch_run"]:
        assert required in names


def test_library_loads_and_exports_every_declared_symbol():
    from minipoa_b200 import _lib

    L = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert missing == []
    # every declared function has a Python signature
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_dp_backend_names_the_cuda_kernel():
    import minipoa_b200 as mp

    assert "sm100a" in mp.dp_backend()


def test_context_without_a_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import minipoa_b200 as mp

    with pytest.raises(mp.PoaError) as e:
        mp.Context()
    assert e.value.code == 3  # POA_ERR_CUDA


def test_missing_library_is_an_error(tmp_path, monkeypatch):
    from minipoa_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()


def test_params_layout_matches_header():
    from minipoa_b200.params import CParams

    # int32 x4, u64 b/f, i32 x2, u64 k/w, i32 x2, u64 x3, f64, u64 x2, i32 x4, two pointers
    assert ctypes.sizeof(CParams) == 4 * 4 + 16 + 8 + 16 + 8 + 24 + 8 + 16 + 16 + 16

"""The C-ABI library loads and exports every entry point include/nsfsi.h declares (no GPU needed)."""
import ctypes
import re

import nsfsi


def declared():
    text = open(nsfsi.HEADER).read()
    return sorted(set(re.findall(r"\b(nsf_[a-z_0-9]+)\s*\(", text)) - {"nsf_status"})


def test_every_declared_symbol_is_exported():
    L = nsfsi.lib()
    names = declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n


def test_abi_version():
    assert nsfsi.lib().nsf_abi_version() == 1


def test_no_device_is_a_loud_cuda_error_here():
    import torch
    if torch.cuda.is_available():
        return
    try:
        nsfsi.Solver(nsfsi.case_path("sphere48"), device=0)
    except nsfsi.NsfError as e:
        assert e.code == 2
    else:
        raise AssertionError("expected NSF_ERR_CUDA without a GPU")

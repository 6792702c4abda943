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


def test_async_download_argument_checks_without_device():
    """nsf_download_async / _wait / _done refuse null arguments and host-only handles before any device work;
    nsf_host_alloc fails loudly without a device and nsf_host_free accepts null."""
    L = nsfsi.lib()
    t, d = ctypes.c_uint64(), ctypes.c_int32()
    buf = (ctypes.c_double * 8)()
    assert L.nsf_download_async(None, 1, buf, ctypes.byref(t)) == 6
    assert L.nsf_download_wait(None, 1) == 6
    assert L.nsf_download_done(None, 1, ctypes.byref(d)) == 6
    s = nsfsi.Solver(nsfsi.case_path("sphere48"), device=-1)
    assert L.nsf_download_async(s.h, 1, buf, None) == 6
    assert L.nsf_download_async(s.h, 1, buf, ctypes.byref(t)) == 7
    assert L.nsf_download_wait(s.h, 1) == 7
    assert L.nsf_download_done(s.h, 1, ctypes.byref(d)) == 7
    s.close()
    p = ctypes.c_void_p()
    assert L.nsf_host_alloc(0, ctypes.byref(p)) == 6 and not p.value
    assert L.nsf_host_alloc(64, None) == 6
    import torch
    if not torch.cuda.is_available():
        assert L.nsf_host_alloc(64, ctypes.byref(p)) == 2 and not p.value
    assert L.nsf_host_free(None) == 0


def test_every_handle_entry_refuses_a_null_handle():
    """Every entry point that takes a solver, ensemble or slab-group handle returns NSF_ERR_ARG for a null
    handle (other arguments null or zero) before any device work; the error-text calls name the null handle
    and the destroy calls accept it."""
    import inspect
    L = nsfsi.lib()
    src = inspect.getsource(nsfsi.lib)
    names = [ln.split('"')[1] for ln in src.splitlines() if ln.strip().startswith('"nsf_')]
    checked = 0
    for n in names:
        f = getattr(L, n)
        args = f.argtypes
        if not args or args[0] is not ctypes.c_void_p or f.restype is not ctypes.c_int32 or n == "nsf_host_free":
            continue
        vals = [None] + [0 if a in (ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t)
                         else 0.0 if a is ctypes.c_double else None for a in args[1:]]
        assert f(*vals) == 6, n
        checked += 1
    assert checked >= 40
    assert b"null" in L.nsf_last_error(None)
    assert b"null" in L.nsf_ensemble_last_error(None)
    assert b"null" in L.nsf_slab_group_last_error(None)
    L.nsf_destroy(None)
    L.nsf_ensemble_destroy(None)
    L.nsf_slab_group_destroy(None)

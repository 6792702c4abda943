"""nsf_step_metrics_noalloc: the allocation-free entry point for callers that cannot let a library call
cudaMalloc (frameworks that own all device memory, code under CUDA stream capture, real-time loops).

It is checked against the solver's own end-of-step metrics (nsf_march's history norms and next dt) on
two consecutive steps, with the tolerances of the parity tests. Collected last on purpose: it shares
a fixed device array with any other caller and is independent of the other tests' state."""
import ctypes

import numpy as np
import pytest

import nsfsi

NORM_TOL = 1e-8  # as in test_parity_gpu.py
DT_TOL = 1e-10


@pytest.mark.gpu
def test_noalloc_metrics_match_the_solver_on_two_consecutive_steps():
    import torch

    cfg = nsfsi.config_load("tests/golden/cases/tgv_small.cfg")
    L = nsfsi.lib()
    with nsfsi.Solver(cfg) as s:
        for call in range(2):
            u_old = s.download(range(5))
            s.march(1)
            s.sync()
            u_new = s.download(range(5))
            norms = s.history()[-1][2:7]
            _, level, dt_next = s.time()
            assert level == call + 1
            d_old = torch.tensor(u_old, device="cuda")
            d_new = torch.tensor(u_new, device="cuda")
            d_out = torch.full((6,), -1.0, dtype=torch.float64, device="cuda")
            st = L.nsf_step_metrics_noalloc(ctypes.byref(cfg), ctypes.c_void_p(d_old.data_ptr()),
                                            ctypes.c_void_p(d_new.data_ptr()), None,
                                            ctypes.c_void_p(d_out.data_ptr()),
                                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert st == 0
            torch.cuda.synchronize()
            out = d_out.cpu().numpy()
            assert np.abs(out[:5] - norms).max() <= NORM_TOL * np.abs(norms).max(), (out[:5], norms)
            assert abs(out[5] / dt_next - 1) <= DT_TOL, (out[5], dt_next)


@pytest.mark.gpu
def test_noalloc_dt_with_the_callers_end_time_clip():
    """An end_time run: the entry point returns the unclipped dt, and the clip the header asks callers to
    apply (dt = t_end - t where t + dt > t_end, Solver.cpp:85-87) gives what the solver records."""
    import torch

    base = nsfsi.config_load("tests/golden/cases/tgv_small.cfg")
    with nsfsi.Solver(base) as s:
        s.march(1)
        t1, _, dt1 = s.time()
    cfg = nsfsi.config_load("tests/golden/cases/tgv_small.cfg")
    cfg.stop_criterion = 1  # end_time
    cfg.t_end = t1 + 0.5 * dt1  # the second step is shortened
    L = nsfsi.lib()
    with nsfsi.Solver(cfg) as s:
        u_old = s.download(range(5))
        s.march(1)
        s.sync()
        u_new = s.download(range(5))
        t, level, dt_next = s.time()
        assert level == 1 and t == t1 and dt_next == cfg.t_end - t
        d_old, d_new = torch.tensor(u_old, device="cuda"), torch.tensor(u_new, device="cuda")
        d_out = torch.full((6,), -1.0, dtype=torch.float64, device="cuda")
        assert L.nsf_step_metrics_noalloc(ctypes.byref(cfg), ctypes.c_void_p(d_old.data_ptr()),
                                          ctypes.c_void_p(d_new.data_ptr()), None, ctypes.c_void_p(d_out.data_ptr()),
                                          None) == 0
        torch.cuda.synchronize()
        dt = float(d_out[5].item())
        assert abs(dt / dt1 - 1) <= DT_TOL  # unclipped: the full limit of the new state
        clipped = cfg.t_end - t if t + dt > cfg.t_end else dt
        assert clipped == dt_next


@pytest.mark.gpu
def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    cfg = nsfsi.config_load("tests/golden/cases/tgv_small.cfg")
    cfg.NI = cfg.NJ = cfg.NK = 320  # 32.8M nodes > 29,826,048
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(d.data_ptr())
    assert nsfsi.lib().nsf_step_metrics_noalloc(ctypes.byref(cfg), p, p, None, p, None) == 6

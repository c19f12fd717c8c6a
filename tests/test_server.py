"""The solve server's host logic on the CPU (no GPU here): argument errors, refusal of a request
larger than the budget, and a request that cannot create its device handle ending as failed,
not hanging the queue."""
import ctypes as C

import numpy as np
import pytest

from itofoggysim_b200 import _native as N, scene as S
from itofoggysim_b200.server import SolveServer


def test_refused_when_larger_than_budget(native):
    with SolveServer(max_concurrent=2, memory_budget=1 << 20) as srv:
        rid = srv.submit(S.random_cluster(20, seed=1, p=6))
        info, x, cs = srv.wait(rid)
        assert info["state"] == N.REQ_REFUSED and info["status"] == N.FOGGY_ERR_NOMEM
        assert x is None and "device bytes" in info["error"]
        srv.release(rid)


def test_failed_without_device(native):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with SolveServer(max_concurrent=1, memory_budget=8 << 30) as srv:
        ids = [srv.submit(S.random_cluster(3, seed=s, p=3)) for s in range(3)]
        for rid in ids:
            info, x, _ = srv.wait(rid)
            assert info["state"] == N.REQ_FAILED and info["status"] == N.FOGGY_ERR_CUDA and x is None
            assert info["ms_latency"] >= 0


def test_request_params_reach_the_handle(native):
    """A request's precision is checked by the handle it runs on: an invalid value fails the
    request with the handle's argument error (raised before any device is needed)."""
    with SolveServer(max_concurrent=2, memory_budget=8 << 30) as srv:
        rid = srv.submit(S.random_cluster(3, seed=1, p=3), precision=7)
        info, x, _ = srv.wait(rid)
        assert info["state"] == N.REQ_FAILED and info["status"] == N.FOGGY_ERR_ARGUMENT and x is None
        assert "precision" in info["error"]


def test_argument_errors(native):
    L = N.load()
    with SolveServer(max_concurrent=1, memory_budget=1 << 20) as srv:
        rid = C.c_int64()
        assert L.foggy_server_submit(srv.h, None, C.byref(rid)) == N.FOGGY_ERR_ARGUMENT
        info = N.FoggyRequestInfo()
        assert L.foggy_server_poll(srv.h, 12345, 0, C.byref(info), None, 0, None) == N.FOGGY_ERR_ARGUMENT
        assert L.foggy_server_cancel(srv.h, 12345) == N.FOGGY_ERR_ARGUMENT
        assert L.foggy_server_release(srv.h, 12345) == N.FOGGY_ERR_ARGUMENT
        sc = S.random_cluster(3, seed=1, p=3)
        bad = sc.param_index.copy()
        bad[0] = 7
        sc.param_index = bad
        with pytest.raises(N.FoggyError):
            srv.submit(sc)
    assert L.foggy_server_start(0, 0, 0, C.byref(C.c_void_p())) == N.FOGGY_ERR_ARGUMENT

"""The solve server on the GPU: a mixed stream of requests (different sphere counts, orders and
right-hand-side counts) run up to three at a time, and every result is bit-identical to the same
request solved alone on a handle of its own (a request's several right-hand sides as one block,
foggy_solve_block, within the tolerance of one-by-one solves); one solve per plane wave matches single-wave solves
and the oracle; a request larger than the budget is refused; a queued request can be cancelled."""
import numpy as np
import pytest

from itofoggysim_b200 import _native as N, scene as S, solver
from itofoggysim_b200.server import SolveServer

pytestmark = pytest.mark.gpu


def _waves(rng, n):
    th = np.arccos(rng.uniform(-1, 1, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    return dict(wave_theta=th, wave_phi=ph, jones=np.tile([1.0, 0.0, 0.0, 0.0], (n, 1)), wave_g=np.ones(n),
                wave_phase=np.zeros(n), wave_d0=np.zeros((n, 3)))


def _stream(k=8):
    rng = np.random.default_rng(5)
    out = []
    for i in range(k):
        n = int(rng.integers(3, 30))
        sc = S.random_cluster(n, seed=100 + i, p=int(rng.integers(3, 9)), waves=_waves(rng, int(rng.integers(1, 4))))
        out.append((sc, bool(i % 2)))
    return out


def test_stream_results_equal_solo_solves(native):
    reqs = _stream()
    with SolveServer(max_concurrent=3) as srv:
        ids = [srv.submit(sc, rhs_per_wave=pw) for sc, pw in reqs]
        got = [srv.wait(rid) for rid in ids]
    for (sc, pw), (info, x, cs) in zip(reqs, got):
        assert info["state"] == N.REQ_DONE, info["error"]
        assert info["ms_latency"] >= info["ms_solve"] > 0 and info["footprint"] > 0
        with solver.MultiSphereSolver(sc) as s:
            if pw and sc.n_waves > 1:
                # several right-hand sides run as one block in the server, as alone
                xs, css, _, _, _ = s.solve_block()
                xr, _, _ = s.solve_rhs()
                for r in range(sc.n_waves):
                    assert np.linalg.norm(xs[r] - xr[r]) <= 1e-6 * np.linalg.norm(xr[r])
            elif pw:
                xs, css, _ = s.solve_rhs()
            else:
                x1, _ = s.solve()
                xs, css = x1[None, :], s.cross_sections(x1)[None, :]
        assert x.shape == xs.shape and np.array_equal(x, xs)
        assert np.array_equal(cs, css)


def test_rhs_per_wave_matches_single_wave_solves_and_oracle(native, oracle):
    rng = np.random.default_rng(9)
    sc = S.random_cluster(6, seed=3, p=5, waves=_waves(rng, 3))
    with solver.MultiSphereSolver(sc) as s:
        xs, css, st = s.solve_rhs()
    assert st["backward_error"] <= sc.gmres_tolerance
    for r in range(3):
        keys = ("wave_theta", "wave_phi", "jones", "wave_g", "wave_phase", "wave_d0")
        one = S.Scene(**{**sc.__dict__, **{k: getattr(sc, k)[r:r + 1] for k in keys}})
        with solver.MultiSphereSolver(one) as s1:
            x1, _ = s1.solve()
            c1 = s1.cross_sections(x1)
        assert np.max(np.abs(xs[r] - x1)) <= 1e-12 * np.max(np.abs(x1))
        assert np.allclose(css[r], c1, rtol=1e-12, atol=1e-12 * abs(c1[1]))
        P = oracle.Problem(one)
        A = np.stack([P.matvec(np.eye(P.n)[i]) for i in range(P.n)], axis=1)
        xr = np.linalg.solve(A, P.vector_b())
        assert np.linalg.norm(xs[r] - xr) <= 1e-6 * np.linalg.norm(xr)


def test_refusal_and_cancel(native):
    big = S.random_cluster(60, seed=2, p=8)
    small = S.random_cluster(4, seed=3, p=3)
    with SolveServer(max_concurrent=1, memory_budget=64 << 20) as srv:
        rid = srv.submit(big)
        info, x, _ = srv.wait(rid)
        assert info["state"] == N.REQ_REFUSED and x is None
    with SolveServer(max_concurrent=1) as srv:
        first = srv.submit(S.random_cluster(120, seed=4, p=10))
        second = srv.submit(small)
        rc = srv.cancel(second)
        info2, _, _ = srv.poll(second)
        if rc == N.FOGGY_OK:
            assert info2["state"] == N.REQ_CANCELLED
        else:   # it had already started
            assert rc == N.FOGGY_ERR_STATE
        info1, x1, _ = srv.wait(first)
        assert info1["state"] == N.REQ_DONE and x1 is not None


def test_handles_created_and_destroyed_beside_a_solve(native):
    """Device memory comes from a stream-ordered pool shared by the handles: handles set up, applied
    and torn down in another thread while a solve runs (their freed blocks going back to the pool and
    out to the next handle) leave the solve's result bit-identical to the same solve alone, and each
    churned handle's operator equals the same operator on a quiet GPU."""
    import threading
    big = S.random_cluster(40, seed=71, p=8)
    small = [S.random_cluster(int(n), seed=200 + i, p=int(p)) for i, (n, p) in enumerate([(5, 4), (12, 6), (20, 7)])]
    with solver.MultiSphereSolver(big) as s:
        x_alone, _ = s.solve()
    ref = []
    for sc in small:
        v = np.random.default_rng(3).standard_normal(sc.vector_length()) + 0j
        with solver.MultiSphereSolver(sc) as s:
            ref.append((v, s.calculate_vector_b(v)))
    errors, done = [], threading.Event()

    def churn():
        try:
            for k in range(30):
                sc = small[k % len(small)]
                v, y_ref = ref[k % len(small)]
                with solver.MultiSphereSolver(sc) as s:
                    if not np.array_equal(s.calculate_vector_b(v), y_ref):
                        errors.append("operator of churned handle %d differs" % k)
        except Exception as e:  # reported by the main thread
            errors.append(repr(e))
        finally:
            done.set()

    t = threading.Thread(target=churn)
    t.start()
    solves = 0
    try:
        while solves < 3 or not done.is_set():
            with solver.MultiSphereSolver(big) as s:
                x, st = s.solve()
            assert st["status"] == 0 and np.array_equal(x, x_alone)
            solves += 1
    finally:
        t.join()
    assert not errors, errors[:3]

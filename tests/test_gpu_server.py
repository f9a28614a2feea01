"""The request server (qcuServer*): continuous batching over resident gauge
configurations.

The central check: every request's solution is the same whether it ran alone
or in a mix where other requests (other lattices, kappas, Wilson and clover,
different RHS counts) join and leave its batch while it iterates. Each
solution is also checked independently with the CPU oracle's full operator:
|b - M x| / |b| below the tolerance (1e-10)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10
EPS = 0.4
LA, LB = (8, 8, 8, 8), (4, 4, 4, 8)


def requests():
    # (config index, kappa, csw, nrhs, source seed)
    return [(0, 0.125, 1.0, 3, 11), (1, 0.130, 0.0, 2, 12), (0, 0.120, 0.0, 1, 13), (2, 0.1375, 1.0, 4, 14),
            (0, 0.133, 1.0, 5, 15), (1, 0.128, 1.0, 1, 16), (0, 0.127, 1.0, 2, 17), (2, 0.121, 0.0, 3, 18)]


CONFIGS = [(LA, 101), (LB, 202), (LA, 303)]


def sources(oracle, L, nrhs, seed):
    return np.stack([oracle.full_spinor_random(L, seed * 100 + r) for r in range(nrhs)])


def true_residual(oracle, x, b, U, L, kappa, csw):
    C = oracle.clover_build(U, L, kappa * csw)
    r = b - oracle.apply_full(x, U, C, L, kappa, -1.0)
    return np.linalg.norm(r) / np.linalg.norm(b)


def make_server(qcu_lib):
    srv = qcu_lib.Server(columns=8, clover_slots=4, tol=TOL)
    ids = [srv.add_config(L, seed, EPS) for L, seed in CONFIGS]
    return srv, ids


def test_results_alone_equal_results_in_the_mix(cuda, qcu_lib, oracle):
    reqs = requests()
    B = [sources(oracle, CONFIGS[c][0], n, sd) for c, _, _, n, sd in reqs]
    srv, ids = make_server(qcu_lib)
    with srv:
        for i in ids:
            srv.prepare(i)
        # the mix: staggered arrivals, so requests join batches that are iterating
        X_mix = [np.zeros_like(b) for b in B]
        arrivals = [0.002 * k for k in range(len(reqs))]
        lat, reps_mix, code = srv.run_trace(arrivals, [ids[c] for c, *_ in reqs], [k for _, k, *_ in reqs],
                                            [w for _, _, w, *_ in reqs], [n for *_, n, _ in reqs], B, X_mix)
        assert code == qcu_lib.QCU_SUCCESS
        assert all(t > 0 for t in lat)
        # each request alone, on an idle server
        for k, (c, kap, csw, n, _) in enumerate(reqs):
            x = np.zeros_like(B[k])
            t = srv.submit(ids[c], kap, csw, n, B[k], x)
            _, reps, code = srv.wait(t, n)
            assert code == qcu_lib.QCU_SUCCESS
            srv.release(t)
            rel = np.linalg.norm(x - X_mix[k]) / np.linalg.norm(x)
            assert rel < 1e-9, (k, rel)
            for ra, rm in zip(reps, reps_mix[k]):
                assert ra["converged"] and rm["converged"]
                assert ra["true_residual"] < TOL and rm["true_residual"] < TOL
            # independent check of the mixed-run solution on the CPU
            L = CONFIGS[c][0]
            U = oracle.gauge_random(L, CONFIGS[c][1], EPS)
            for r in range(n):
                assert true_residual(oracle, X_mix[k][r], B[k][r], U, L, kap, csw) < TOL


def test_submit_poll_query_lifecycle(cuda, qcu_lib, oracle):
    srv, ids = make_server(qcu_lib)
    with srv:
        b = sources(oracle, LB, 2, 5)
        x = np.zeros_like(b)
        t = srv.submit(ids[1], 0.126, 1.0, 2, b, x)
        assert srv.pending == 1
        fin, *_ = srv.query(t, 2)
        assert not fin
        lat, reps, code = srv.wait(t, 2)
        assert code == qcu_lib.QCU_SUCCESS and lat > 0 and srv.pending == 0
        assert all(r["converged"] for r in reps)
        srv.release(t)
        with pytest.raises(qcu_lib.QcuError):
            srv.release(t)
        assert srv.device_bytes > 0


def test_request_larger_than_the_batch_is_rejected(cuda, qcu_lib, oracle):
    srv, ids = make_server(qcu_lib)
    with srv:
        b = sources(oracle, LB, 9, 6)
        with pytest.raises(qcu_lib.QcuError) as e:
            srv.submit(ids[1], 0.126, 1.0, 9, b, np.zeros_like(b))
        assert e.value.code == qcu_lib.QCU_ERR_INVALID_ARG


def test_nan_source_fails_only_its_request(cuda, qcu_lib, oracle):
    srv, ids = make_server(qcu_lib)
    with srv:
        good = sources(oracle, LB, 1, 7)
        bad = sources(oracle, LB, 1, 8)
        bad[0, 0, 3, 1, 2] = np.nan
        xg, xb = np.zeros_like(good), np.zeros_like(bad)
        tb = srv.submit(ids[1], 0.125, 1.0, 1, bad, xb)
        tg = srv.submit(ids[1], 0.125, 1.0, 1, good, xg)
        _, _, code_b = srv.wait(tb, 1)
        _, reps, code_g = srv.wait(tg, 1)
        assert code_b == qcu_lib.QCU_ERR_INVALID_ARG
        assert code_g == qcu_lib.QCU_SUCCESS and reps[0]["converged"]


def test_small_budget_evicts_idle_configurations(cuda, qcu_lib, oracle):
    # room for about one 8^4 configuration: the second one evicts the first
    srv = qcu_lib.Server(columns=4, clover_slots=2, tol=TOL, device_budget=200 << 20)
    with srv:
        a = srv.add_config(LA, 101, EPS)
        c = srv.add_config(LA, 303, EPS)
        for cid, seed in ((a, 101), (c, 303), (a, 101)):
            b = sources(oracle, LA, 1, 9)
            x = np.zeros_like(b)
            t = srv.submit(cid, 0.124, 1.0, 1, b, x)
            _, reps, code = srv.wait(t, 1)
            assert code == qcu_lib.QCU_SUCCESS
            U = oracle.gauge_random(LA, seed, EPS)
            assert true_residual(oracle, x[0], b[0], U, LA, 0.124, 1.0) < TOL
        assert srv.device_bytes <= 200 << 20

"""The serving loop (lbm_server_*): a request queue over one batch.

- early retirement: a request with a residual tolerance retires at the first
  check (every check_every steps) whose density residual sum |rho_k -
  rho_(k-1)| (the quantity kernel.cu:232-248 prints) is at most the
  tolerance, and its result is bit for bit the same domain run alone for
  the same number of steps;
- a request without a tolerance runs its whole budget and equals the domain
  alone (16-bit storage included: batch members use the per-node layout,
  which gives the same bits as the paired default);
- admission: FIFO stops at the first request that does not fit the pool,
  SHORTEST admits the least work first and skips what does not fit; the
  backlog horizon limits the work resident at once;
- a request that can never fit is refused at submit.
"""
import numpy as np
import pytest

import oracle_lib as O

pkg = O.pkg
pytestmark = pytest.mark.gpu


def cavity(n, re=100.0, mrt=False, les=False):
    return pkg.make_inputval(n, casetype=pkg.CAVITY, re=re, u=0.1, mrt=mrt, les=les,
                             cs=0.1 if les else 0.0, h=n)


def opts(storage=pkg.STORE_F32, seed=5):
    return pkg.default_options(storage=storage, init_kind=pkg.INIT_DENSITY_NOISE,
                               noise_amp=1e-6, seed=seed)


def alone_fields(iv, o, steps):
    d = pkg.Domain(iv, o)
    d.run(steps)
    m = d.macroscopic()
    d.close()
    return m


def assert_fields_equal(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_early_retirement_at_the_residual_tolerance():
    iv = cavity(32)
    o = opts()
    every, horizon = 64, 2048
    # residual alone after every check interval
    d = pkg.Domain(iv, o)
    res = []
    for _ in range(horizon // every):
        d.run(every)
        res.append(float(d.diagnostics()[4]))
    d.close()
    tol = 1.5 * res[-1]
    first = next(k for k, r in enumerate(res) if r <= tol)
    want_steps = every * (first + 1)
    s = pkg.Server(hbm_budget=256 << 20, chunk_steps=32, check_every=every)
    i = s.submit(iv, o, steps=100000, tol=tol)
    s.wait(i)
    info = s.info(i)
    assert info["state"] == pkg.REQ_DONE and info["converged"] == 1
    assert info["steps_done"] == want_steps, (info, res)
    assert info["residual"] <= tol
    assert abs(info["residual"] - res[first]) <= 1e-9 * max(1.0, res[first])
    assert 0 <= info["t_arrive"] <= info["t_admit"] <= info["t_done"]
    got = s.result(i)
    assert_fields_equal(got, alone_fields(iv, o, want_steps))
    st = s.stats()
    assert st["completed"] == 1 and st["converged"] == 1 and st["resident"] == 0
    assert st["executed_lups"] == pytest.approx(32 ** 3 * want_steps)
    s.release(i)
    s.close()


@pytest.mark.parametrize("storage", [pkg.STORE_F32, pkg.STORE_F16_SHIFT, pkg.STORE_BF16_SHIFT])
def test_budget_run_equals_alone(storage):
    iv = cavity(40, re=300.0, mrt=True, les=True)
    o = opts(storage)
    s = pkg.Server(hbm_budget=256 << 20, chunk_steps=16)
    i = s.submit(iv, o, steps=150)
    s.wait(i)
    assert s.info(i)["steps_done"] == 150 and s.info(i)["converged"] == 0
    assert_fields_equal(s.result(i), alone_fields(iv, o, 150))
    s.close()


def _admission(policy, horizon=0.0):
    big, small = cavity(64), cavity(16)
    o = opts()
    nb = pkg.batch_domain_bytes(big, o)
    assert pkg.batch_domain_bytes(small, o) * 5 < nb
    s = pkg.Server(hbm_budget=int(2.5 * nb), chunk_steps=32, policy=policy,
                   backlog_horizon_s=horizon, nominal_mlups=1000.0 if horizon else 0.0)
    used0 = s.stats()["pool_used_bytes"]
    ids = [s.submit(big, o, steps=64) for _ in range(3)]
    ids += [s.submit(small, o, steps=96) for _ in range(2)]
    s.progress()
    states = [s.info(i)["state"] for i in ids]
    for _ in range(100000):
        if all(s.info(i)["state"] == pkg.REQ_DONE for i in ids):
            break
        s.progress()
    for i in ids:
        assert s.info(i)["steps_done"] == (64 if i in ids[:3] else 96)
    st = s.stats()
    assert st["completed"] == 5 and st["queued"] == 0 and st["resident"] == 0
    assert st["tts_p50_s"] <= st["tts_p99_s"]
    assert st["service_p50_s"] <= st["service_p99_s"]
    assert st["pool_used_bytes"] == used0
    res = (s, ids, big, small, o)
    return states, res


def test_fifo_admission_has_no_overtaking():
    states, (s, ids, big, small, o) = _admission(pkg.SERVE_FIFO)
    R, Q = pkg.REQ_RESIDENT, pkg.REQ_QUEUED
    assert states == [R, R, Q, Q, Q], states
    # arrival order is admission order
    t = [s.info(i)["t_admit"] for i in ids]
    assert t == sorted(t)
    assert_fields_equal(s.result(ids[2]), alone_fields(big, o, 64))
    s.close()


def test_shortest_first_admission_skips_what_does_not_fit():
    states, (s, ids, big, small, o) = _admission(pkg.SERVE_SHORTEST)
    R, Q = pkg.REQ_RESIDENT, pkg.REQ_QUEUED
    assert states == [R, R, Q, R, R], states
    # the small requests were admitted first, the third big one last
    assert s.info(ids[4])["t_admit"] <= s.info(ids[0])["t_admit"]
    assert s.info(ids[2])["t_admit"] >= s.info(ids[1])["t_admit"]
    assert_fields_equal(s.result(ids[4]), alone_fields(small, o, 96))
    s.close()


def test_backlog_horizon_limits_resident_work():
    # a horizon far below one request's work admits one request at a time
    states, (s, ids, big, small, o) = _admission(pkg.SERVE_FIFO, horizon=1e-9)
    R, Q = pkg.REQ_RESIDENT, pkg.REQ_QUEUED
    assert states == [R, Q, Q, Q, Q], states
    s.close()


def test_submit_refuses_what_can_never_fit():
    iv, o = cavity(64), opts()
    nb = pkg.batch_domain_bytes(iv, o)
    s = pkg.Server(hbm_budget=nb // 2, chunk_steps=32)
    with pytest.raises(pkg.LbmError) as e:
        s.submit(iv, o, steps=10)
    assert e.value.code == pkg.LBM_ERR_BUDGET
    with pytest.raises(pkg.LbmError) as e:
        s.submit(cavity(8), o, steps=0)
    assert e.value.code == pkg.LBM_ERR_INVALID
    with pytest.raises(pkg.LbmError) as e:
        s.result(12345)
    assert e.value.code == pkg.LBM_ERR_INVALID
    i = s.submit(cavity(8), o, steps=4)
    with pytest.raises(pkg.LbmError) as e:
        s.release(i)  # not done yet
    assert e.value.code == pkg.LBM_ERR_STATE
    s.wait(i)
    s.release(i)
    s.close()

"""Error paths on the GPU: bad input states, a poisoned request inside a batch, and the bounded
device wait of the table staging running out. The reference exits the process on errors
(gpu_utils.cuh:28-48, closest_approach.cu:51-81) and propagates non-finite states into NaNs; this
build returns status codes, and one bad object or request does not spoil the others."""
import numpy as np
import pytest

from gpu_util import dev, host

pytestmark = pytest.mark.gpu

START = (2024, 1, 1, 0, 0, 0.0)


def test_host_inputs_with_bad_states_are_refused():
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    ctx = G.Context()
    r, v = orbits.leo(8, 3)
    for dr, dv in [((np.nan, 0, 0), None), (None, (0, np.inf, 0)), ("origin", None)]:
        rb, vb = r.copy(), v.copy()
        if dr == "origin":
            rb[5] = 0.0
        elif dr is not None:
            rb[5] = dr
        if dv is not None:
            vb[5] = dv
        with pytest.raises(G.GpopError) as e:
            ctx.propagate(START, 30.0, 10, rb, vb)
        assert e.value.status == 1 and "object 5" in str(e.value)
    # the context stays usable
    ro, _ = ctx.propagate(START, 30.0, 10, r, v)
    assert np.isfinite(ro).all()
    # closest approach and the derivative entry points refuse them too
    rb = r.copy()
    rb[2, 1] = np.nan
    with pytest.raises(G.GpopError) as e:
        ctx.closest_approach(START, 30.0, rb, v, np.array([0] * 4 + [1] * 4, np.uint32))
    assert e.value.status == 1
    with pytest.raises(G.GpopError) as e:
        ctx.stm(START, 30.0, 4, rb, v)
    assert e.value.status == 1
    ctx.close()


def test_device_inputs_with_bad_states_fail_alone():
    """On the device path the startup kernel flags the state; the call fails, and every other
    object is propagated exactly as in a clean run."""
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r0, v0 = orbits.mixed_population(64, 5)
    for precision in (G.FP64, G.MIXED):
        ctx = G.Context(precision=precision)
        rc, vc = dev(r0), dev(v0)
        ctx.propagate_device(START, 30.0, 40, rc, vc)
        for bad in ("nan", "origin"):
            rb, vb = r0.copy(), v0.copy()
            if bad == "nan":
                vb[17, 2] = np.nan
            else:
                rb[17] = 0.0
            rd, vd = dev(rb), dev(vb)
            with pytest.raises(G.GpopError) as e:
                ctx.propagate_device(START, 30.0, 40, rd, vd)
            assert e.value.status == 1 and "origin" in str(e.value)
            keep = np.arange(64) != 17
            assert np.array_equal(host(rd)[keep], host(rc)[keep])
            assert np.array_equal(host(vd)[keep], host(vc)[keep])
        # the gravity entry point flags a position at the origin as well
        acc = dev(np.zeros((2, 3)))
        with pytest.raises(G.GpopError) as e:
            ctx.gravity(dev(np.array([[7.0e6, 0.0, 0.0], [0.0, 0.0, 0.0]])), acc, None,
                        precision=precision)
        assert e.value.status == 1
        ctx.close()


def test_bad_state_fails_alone_in_the_split_block():
    """At 40,000 objects the startup and the GJ8 steps run in the split block (5 owner warps per
    SM): a bad state still fails the call, and every other object matches a clean run bit for
    bit."""
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    n = 40000
    assert G.split_block(n) == 5
    r0, v0 = orbits.mixed_population(n, 6)
    for precision in (G.FP64, G.MIXED):
        ctx = G.Context(precision=precision)
        rc, vc = dev(r0), dev(v0)
        ctx.propagate_device(START, 30.0, 12, rc, vc)
        rb = r0.copy()
        rb[23456] = 0.0
        rd, vd = dev(rb), dev(v0)
        with pytest.raises(G.GpopError) as e:
            ctx.propagate_device(START, 30.0, 12, rd, vd)
        assert e.value.status == 1
        keep = np.arange(n) != 23456
        assert np.array_equal(host(rd)[keep], host(rc)[keep])
        assert np.array_equal(host(vd)[keep], host(vc)[keep])
        ctx.close()


def test_poisoned_request_fails_alone_in_a_batch():
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    reqs = orbits.batch_requests(12, 77, max_days=0.05)
    clean = [dict(q) for q in reqs]
    poisoned = [dict(q) for q in reqs]
    r3 = poisoned[3]["r"].copy()
    r3[0, 0] = np.nan
    poisoned[3]["r"] = r3
    poisoned[7]["h"] = 0.0
    r9 = poisoned[9]["r"].copy()
    r9[-1] = 0.0
    poisoned[9]["r"] = r9
    bad = (3, 7, 9)
    ctx = G.Context(precision=G.MIXED)
    good = [q for i, q in enumerate(clean) if i not in bad]
    expect = ctx.propagate_batch(good)
    out, status, st, msg = ctx.propagate_batch_status(poisoned)
    assert st == 1 and "request 3" in msg and "3 of 12" in msg
    assert status.tolist() == [1 if i in bad else 0 for i in range(12)]
    assert all(out[i] is None for i in bad)
    got = [o for i, o in enumerate(out) if i not in bad]
    for (ra, va), (rb, vb) in zip(expect, got):
        assert np.array_equal(ra, rb) and np.array_equal(va, vb)
    # the plain entry point refuses the same requests and still propagates the others
    with pytest.raises(G.GpopError) as e:
        ctx.propagate_batch(poisoned)
    assert e.value.status == 1
    ctx.close()


def test_staging_wait_gives_up_and_reports(monkeypatch):
    """A context made with the test setting GPOP_TEST_FIRST_WAIT_SPINS=0 gives its first staging
    wait no polls: every block raises the timeout, waits (bounded) for the copy it issued, and
    leaves. The call returns GPOP_ERR_TIMEOUT and reports that every copy had landed before its
    block left. A context made without the setting works as usual afterwards."""
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r0, v0 = orbits.leo(256, 9)
    monkeypatch.setenv("GPOP_TEST_FIRST_WAIT_SPINS", "0")
    ctx = G.Context()
    monkeypatch.delenv("GPOP_TEST_FIRST_WAIT_SPINS")
    for _ in range(2):
        with pytest.raises(G.GpopError) as e:
            ctx.propagate_device(START, 30.0, 8, dev(r0), dev(v0))
        assert e.value.status == 5
        assert "every copy had landed" in str(e.value)
    ctx.close()
    ctx = G.Context()
    r, v = dev(r0), dev(v0)
    ctx.propagate_device(START, 30.0, 8, r, v)
    assert np.isfinite(host(r)).all()
    ctx.close()

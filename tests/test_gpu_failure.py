"""Failure detection on the GPU without a fault.

Every device wait in the kernels is bounded; when one runs out the kernel
sets the session's error word and returns, and the host turns the word into
GPUM_ERR_DEVICE.  The self-test entry point makes such a wait run out on
purpose (an mbarrier that nothing arrives on, polled a bounded number of
times and for at most 50 ms), so this test sees the status a lost TMA tile
or tensor-core commit would produce, and then checks that the session keeps
working: the same run before and after gives the same chains.
"""
import numpy as np
import pytest

from gpumetropolis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_device_error_and_session_recovers(gpu):
    w = W.make("gaussian", n_obs=2000)
    m = w.model
    C = 8
    init = np.linspace(3.0, 3.8, C).reshape(C, 1)
    sd = np.full((C, 1), 0.05)
    with gpu.Session(m.loglik.code, m.loglik.consts, m.prior.code, m.prior.consts, 1, w.data,
                     1, w.n_obs) as s:
        d1, a1, l1 = s.run(init, sd, np.ones(C), 64, 3, 0)
        for polls in (1, 4096):
            with pytest.raises(gpu.GpumError) as e:
                s.selftest_wait(polls)
            assert e.value.code == gpu.ERR_DEVICE
            assert "device-side failure" in str(e.value)
        d2, a2, l2 = s.run(init, sd, np.ones(C), 64, 3, 0)
        assert np.array_equal(d1, d2) and np.array_equal(a1, a2) and np.array_equal(l1, l2)
        got = s.loglik_batch(init)
    ref = -((w.data[:, 0][None, :] - init) ** 2).sum(axis=1) / 8
    np.testing.assert_allclose(got, ref, rtol=1e-6)

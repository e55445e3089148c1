"""Device-side failure detection without a GPU fault: a bounded mbarrier wait
that nothing completes gives up, the kernel sets the handle's error word and
returns, and the host call reports REMC_ERR_TIMEOUT. The handle (and the CUDA
context) stays usable: the next calls succeed and give the same energies."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_handle_recovers(built_lib):
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200._capi import REMC_ERR_TIMEOUT, RemcError, check, lib
    from remcdockingsimulator_b200.engine import Engine
    w = synth.crowded(3)
    with Engine(w.systems, 4, w.params) as eng:
        e0 = eng.energy_full()
        for _ in range(2):  # twice: the error word is cleared after it is reported
            with pytest.raises(RemcError) as exc:
                check(lib().remc_check_wait_timeout(eng._h, 4096))
            assert exc.value.code == REMC_ERR_TIMEOUT
            assert "gave up" in str(exc.value)
            e1 = eng.energy_full()  # a device error would fail every later call
            assert np.array_equal(e0, e1)
        check(lib().remc_sync(eng._h))
        with pytest.raises(RemcError):
            check(lib().remc_check_wait_timeout(eng._h, 0))  # polls out of range

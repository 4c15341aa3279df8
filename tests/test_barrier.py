"""The bounded grid barrier of the persistent CG kernels (tf_barrier_check).

A barrier whose wait can never complete (more arrivals expected than blocks
launched: a flag that nothing sets) must end the launch with status 2 after
its time limit, with the GPU context still usable; a complete barrier must
report 0.  The failure is made by the arguments, never by a fault."""
import pytest

import tetfit_b200 as tb


@pytest.mark.parametrize("args", [
    dict(blocks=0, expected=1), dict(blocks=4, expected=0), dict(blocks=4, expected=9),
    dict(blocks=4, expected=4, rounds=0), dict(blocks=4, expected=4, timeout_us=0),
    dict(blocks=4, expected=4, timeout_us=2_000_000),
])
def test_barrier_check_rejects_bad_arguments(product_lib, args):
    with pytest.raises(tb.TetfitError) as e:
        tb.barrier_check(**args)
    assert e.value.code == tb.TF_E_ARG
    assert "tf_barrier_check" in tb.last_thread_error()


@pytest.mark.gpu
def test_barrier_completes_on_every_sm(product_lib):
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    status, ms = tb.barrier_check(sms, sms, rounds=2000, timeout_us=100000)
    assert status == 0
    # one barrier of a full grid takes microseconds, far from the limit
    assert ms / 2000 < 0.1


@pytest.mark.gpu
def test_barrier_wait_that_cannot_complete_reports_status(product_lib):
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    status, ms = tb.barrier_check(sms, sms + 1, rounds=50, timeout_us=20000)
    assert status == 2
    # the first wait runs out (20 ms); every later barrier falls through
    assert 19.0 <= ms < 1000.0
    # the context is still usable: a complete barrier right after
    status, _ = tb.barrier_check(8, 8, rounds=10)
    assert status == 0

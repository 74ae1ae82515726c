"""Failure detection without faulting the GPU.

* A lost TMA copy: ts_context_inject_fault(TS_FAULT_SKIP_COPY, plane) makes the producers of
  the next fused stage launch skip one plane's copy, with every mbarrier wait of that launch
  bounded to 1 ms. The consumers that needed the plane give up, record the timeout in the
  device error word and return; ts_context_sync reports TS_ERR_DEVICE (and clears the word),
  and the next run on the same context is clean and matches an untouched run bitwise.
* Allocation failure injected on the host (TS_FAULT_ALLOC) and a real one (a domain larger
  than the device) surface as TS_ERR_OUT_OF_MEMORY; the context stays usable.
* A NaN or infinite state (NaN from the initial-condition expression, infinity set by the
  caller) is reported by ts_integrator_check_finite as TS_ERR_NONFINITE.
Every wait in these launches is bounded; nothing traps, faults or hangs.
"""
import numpy as np
import pytest

import treesap_b200 as tsb
from treesap_b200.configs import c2_pulses, wave_desc

pytestmark = pytest.mark.gpu
TS_ERR_OUT_OF_MEMORY, TS_ERR_DEVICE, TS_ERR_NONFINITE = 4, 5, 7


def c2_like(precision=tsb.TS_F64, scheme=tsb.TS_RK4):
    return wave_desc((48, 40, 36), 4, periodic=(0, 0, 0), ko=0.2, abl_thickness=6, abl_max=10.0,
                     bc=tsb.TS_BC_DIRICHLET, precision=precision, scheme=scheme)


def clean_run(ctx, desc, steps):
    it = tsb.Integrator(ctx, desc)
    it.initialise(tsb.TS_INIT_GAUSSIAN, c2_pulses(5, 4))
    it.step(steps)
    out = it.get_state()
    ctx.sync()
    it.close()
    return out


@pytest.mark.parametrize("precision,scheme", [(tsb.TS_F64, tsb.TS_RK4), (tsb.TS_F32_STAGE, tsb.TS_RK4),
                                              (tsb.TS_F64, tsb.TS_EULER)])
@pytest.mark.parametrize("plane", [0, 5, 11])
def test_lost_copy_is_reported_and_the_context_recovers(ctx, precision, scheme, plane):
    desc = c2_like(precision, scheme)
    want = clean_run(ctx, desc, 3)

    it = tsb.Integrator(ctx, desc)
    it.initialise(tsb.TS_INIT_GAUSSIAN, c2_pulses(5, 4))
    ctx.inject_fault(tsb.TS_FAULT_SKIP_COPY, plane)
    it.step(1)  # the first stage launch of this step loses one plane's copy
    with pytest.raises(tsb.TSError) as e:
        ctx.sync()
    assert e.value.status == TS_ERR_DEVICE
    assert "mbarrier wait timed out" in str(e.value)
    ctx.sync()  # the error word was cleared by the report

    # the same context and integrator run clean afterwards
    it.initialise(tsb.TS_INIT_GAUSSIAN, c2_pulses(5, 4))
    it.step(3)
    got = it.get_state()
    ctx.sync()
    it.close()
    assert np.array_equal(got, want)


def test_injected_fault_is_one_shot_and_clearable(ctx):
    desc = c2_like()
    ctx.inject_fault(tsb.TS_FAULT_SKIP_COPY, 3)
    ctx.inject_fault(tsb.TS_FAULT_NONE)  # cleared before any launch took it
    want = clean_run(ctx, desc, 2)
    got = clean_run(ctx, desc, 2)
    assert np.array_equal(got, want)
    with pytest.raises(tsb.TSError) as e:
        ctx.inject_fault(tsb.TS_FAULT_SKIP_COPY, -1)
    assert e.value.status == 1


def test_injected_allocation_failure_surfaces_as_out_of_memory(ctx):
    desc = c2_like()
    ctx.inject_fault(tsb.TS_FAULT_ALLOC, 1)
    with pytest.raises(tsb.TSError) as e:
        tsb.Integrator(ctx, desc)
    assert e.value.status == TS_ERR_OUT_OF_MEMORY
    # a failure later in the constructor (the third field) as well
    ctx.inject_fault(tsb.TS_FAULT_ALLOC, 3)
    with pytest.raises(tsb.TSError) as e:
        tsb.Integrator(ctx, c2_like(tsb.TS_F32_STAGE))
    assert e.value.status == TS_ERR_OUT_OF_MEMORY
    ctx.inject_fault(tsb.TS_FAULT_NONE)
    out = clean_run(ctx, desc, 1)
    assert np.isfinite(out).all()


def test_real_allocation_failure_surfaces_as_out_of_memory(ctx):
    """Two 6000^3 FP64 fields (3.5 TB each) cannot be allocated: cudaMalloc refuses at once."""
    with pytest.raises(tsb.TSError) as e:
        tsb.Integrator(ctx, wave_desc(6000, 2))
    assert e.value.status == TS_ERR_OUT_OF_MEMORY
    assert np.isfinite(clean_run(ctx, c2_like(), 1)).all()


def test_nan_in_the_initial_condition_is_reported(ctx):
    desc = wave_desc((24, 20, 16), 2, ko=0.1)
    it = tsb.Integrator(ctx, desc)
    it.initialise_expressions(["exp(-(x^2+y^2+z^2)/0.1^2)", "0.0"])
    it.check_finite()  # a finite state passes
    it.initialise_expressions(["exp(-(x^2+y^2+z^2)/0.1^2) + if(x > 0.5, sqrt(-1), 0)", "0.0"])
    with pytest.raises(tsb.TSError) as e:
        it.check_finite()
    assert e.value.status == TS_ERR_NONFINITE
    it.step(2)  # NaN spreads through the stencils; still reported after stepping
    with pytest.raises(tsb.TSError) as e:
        it.check_finite()
    assert e.value.status == TS_ERR_NONFINITE
    it.close()


def test_infinite_value_set_by_the_caller_is_reported(ctx):
    desc = wave_desc((24, 20, 16), 2)
    it = tsb.Integrator(ctx, desc)
    s = np.zeros(desc.shape())
    s[1, 3, 4, 5] = np.inf
    it.set_state(s)
    with pytest.raises(tsb.TSError) as e:
        it.check_finite()
    assert e.value.status == TS_ERR_NONFINITE
    s[1, 3, 4, 5] = 1.0
    it.set_state(s)
    it.check_finite()
    it.close()

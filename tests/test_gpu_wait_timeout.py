"""The bounded device wait of the z pass, made to run out without any fault.

The z pass stages Green-spectrum columns into shared memory with bulk copies completed on
an mbarrier, and polls that barrier a bounded number of times.  The test-only context
option OSC_OPT_TEST_WAIT_TIMEOUT arms the barrier with the expected byte count but issues
no copy and lowers the poll limit to 64, so nothing is ever in flight, every CTA's wait
gives up, records the fault and returns.  The host must report OSC_E_TIMEOUT, and the next
ordinary call on the same context must succeed and match the FP64 oracle.
"""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200 import native
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu


def _rho(oracle, n):
    x, y, z = gendist(50_000, sigma=(1e-3, 1e-3, 1e-3), seed=31)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    rho, _ = oracle.depose_rho_scalar(x, y, z, 1e-9 / len(x), (1, 1, 1), n, delta, umin)
    return rho, delta


# z lengths 128 and 256: the radix-8 warp engine; 512: the one-exchange engine
@pytest.mark.parametrize("n", [(16, 16, 64), (24, 20, 128), (12, 12, 256)])
def test_z_pass_wait_times_out_then_context_recovers(oracle, n):
    rho, delta = _rho(oracle, n)
    gamma = 2.5
    e_ref, _ = oracle.freespace_solver2(rho, gamma, delta)
    with osc.Context(0) as ctx:
        ctx.set_option(native.OPT_TEST_WAIT_TIMEOUT, 1)
        assert ctx.get_option(native.OPT_TEST_WAIT_TIMEOUT) == 1
        with pytest.raises(osc.OscError) as ei:
            osc.osc_freespace_solver2(ctx, rho, gamma, delta, precision=osc.PREC_FP32)
        assert ei.value.code == native.OSC_E_TIMEOUT
        assert "device wait gave up" in str(ei.value)
        ctx.set_option(native.OPT_TEST_WAIT_TIMEOUT, 0)
        e, _ = osc.osc_freespace_solver2(ctx, rho, gamma, delta, precision=osc.PREC_FP32)
        mx, rm = field_err(e, e_ref)
        assert mx <= 1e-5, (mx, rm)

"""GPU: the bounded mbarrier wait of the V apply's coefficient copies gives up, flags
and returns (no fault, no hang), and the device stays usable afterwards.

The wait runs out on a phase that nothing completes (16 transaction bytes expected,
no copy issued), with a limit of 1e6 SM cycles (about half a millisecond)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _selftest(cycles, complete):
    from vpfhf_b200 import _abi
    out = ctypes.c_int(-1)
    rc = _abi.lib().vfgpu_wait_selftest(ctypes.c_longlong(cycles), complete, ctypes.byref(out))
    assert rc == 0
    return out.value


def test_wait_gives_up_and_flags(cuda):
    assert _selftest(1_000_000, 0) == 1


def test_completed_phase_does_not_flag(cuda):
    assert _selftest(1_000_000, 1) == 0


def test_bad_arguments_refused(cuda):
    from vpfhf_b200 import _abi
    out = ctypes.c_int(0)
    assert _abi.lib().vfgpu_wait_selftest(ctypes.c_longlong(-1), 0, ctypes.byref(out)) == -1
    assert _abi.lib().vfgpu_wait_selftest(ctypes.c_longlong(10**10), 0, ctypes.byref(out)) == -1


def test_device_usable_after_a_timed_out_wait(cuda):
    """After the wait gave up, a V solve (whose applies use the same wait) runs and its
    coefficient copies complete without the flag being set."""
    import vpfhf_b200 as vg
    assert _selftest(1_000_000, 0) == 1
    n, L = 17, 4.0
    h = L / (n - 1)
    ctx = vg.VFContext((n, n, n), (L, L, L), dict(E=1e10, nu=0.25, Gc=100.0), epsilon=2 * h,
                       eta=1e-8, atnum=1, pressurize=True)
    ctx.set_bc(vg.rollers())
    ctx.set_field("pressure", np.full(ctx.N, 1e6))
    ctx.init_cracks([dict(center=(2.0, 2.0, 2.0), r=0.8, theta=0.0, phi=0.0, thickness=2 * h)])
    ctx.time_step_prepare()
    rc, err, su, sv = ctx.am_step()
    assert rc == 0 and su["reason"] > 0 and sv["reason"] > 0, (su, sv)
    ctx.close()

"""Device memory kept across contexts (marked gpu): a context created in the
memory of a destroyed one, and after flash_hy_release_memory, steps bit for
bit as the oracle does (kept blocks hold stale data: nothing may rely on
fresh memory)."""
import numpy as np
import pytest

from flash5_b200 import abi
from flash5_b200.hydro import Hydro, next_dt
from oracle import orc
from tests.cases import make_case


def _run(case, steps=3):
    grid, unk, params = make_case(case)
    ref = unk.copy()
    o = orc.Oracle(params, grid)
    o.eos_init(ref)
    h = Hydro(params, grid)
    h.upload(unk)
    dt, _ = h.compute_dt()
    t, dt_old = 0.0, dt
    for _ in range(steps):
        h(t + dt, dt, dt_old)
        assert o.hydro(ref, t + dt, dt, dt_old) == 0
        t += dt
        dts, _ = h.compute_dt()
        dt_old, dt = dt, next_dt(dts, dt)
    out = grid.new_unk()
    h.download(out)
    return h, grid.interior(out), grid.interior(ref)


@pytest.mark.gpu
def test_contexts_in_kept_memory_match_oracle():
    lib = abi.load_library()
    h, a, b = _run("kh3d")                     # the larger context: its memory is kept when destroyed
    assert np.array_equal(a, b)
    h.close()
    h, a, b = _run("sod3d_rot")                # smaller: takes kept blocks holding the old state
    assert np.array_equal(a, b)
    assert lib.flash_hy_release_memory(-1) == 0   # with a live context: only kept blocks go
    h2, a2, b2 = _run("kh2d_16")
    assert np.array_equal(a2, b2)
    h.close()
    h2.close()
    assert lib.flash_hy_release_memory(0) == 0

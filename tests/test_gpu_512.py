"""Oracle parity at the benchmark's full size: the two-state shock at 512^3
cells, FP64, 4 steps (both sweep orders, the summary after the last step).
The fused native step (the path bench.py times) must give the oracle's dt
sequence bit for bit, every one of the 19 fields bit for bit (halos
included), and the summaries to 1e-12. The oracle's chunk stays in host
memory and the fields are compared one array at a time (about 37 GB of host
memory in all).
"""
import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import oracle_lib as O

pytestmark = pytest.mark.gpu

N, STEPS = 512, 4
STATES = [
    dict(density=0.2, energy=1.0),
    dict(density=1.0, energy=2.5, geometry="cuboid", xmin=0.0, xmax=5.0, ymin=0.0, ymax=2.0,
         zmin=0.0, zmax=2.0),
]


def _mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def test_512_cubed_bitwise_against_the_oracle():
    need = 31 * (N + 5) ** 3 * 8 + 3 * (N + 5) ** 3 * 8
    if _mem_available() < need:
        pytest.skip("host memory below the %.0f GB the 512^3 oracle needs" % (need / 1e9))
    d = dict(x_cells=N, y_cells=N, z_cells=N, xmin=0.0, ymin=0.0, zmin=0.0, xmax=10.0,
             ymax=10.0, zmax=10.0, initial_timestep=0.04, max_timestep=0.04, timestep_rise=1.5,
             end_step=STEPS, end_time=1.0e6, summary_frequency=10, states=STATES)
    ref = O.KeptRun(d)
    try:
        assert ref.steps == STEPS
        kw = {k: v for k, v in d.items() if k != "states"}
        ch = C.Chunk(C.Deck.from_values(states=STATES, **kw))
        try:
            assert ch.run() == STEPS
            assert ch.status == 0
            assert np.array_equal(ch.dt_history(), ref.dt)
            sums, sst = ch.summaries()
            assert np.array_equal(sst, ref.summary_steps)
            np.testing.assert_allclose(sums, ref.summaries, rtol=1e-12, atol=0)
            for n in O.FIELD_NAMES:
                f = ch.field(n)
                r = ref.field(n)
                if not np.array_equal(f, r):
                    bad = np.argwhere(f != r)
                    raise AssertionError("%s differs at %d elements, first %s" %
                                         (n, len(bad), bad[0]))
                del f, r
        finally:
            ch.close()
    finally:
        ref.close()

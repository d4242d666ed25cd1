"""The oracle against golden vectors produced by the reference itself
(wave_CPU.cpp and the reference's flow/sediment kernels run on the CPU)."""
import numpy as np
import pytest

import golden_replay as gr
from pyoracle import Oracle


@pytest.mark.parametrize("name", sorted(gr.CASES))
def test_oracle_matches_reference_golden(name):
    p, o, g = gr.setup(Oracle, name)
    gr.start_step(o, p)
    # boundary interpolation as wavebnd does; dt and time stay as set
    o.call("wave_boundary")
    for tag, call, outs in gr.PHASES:
        o.call(call)
        for f in outs:
            a, b = o.get(f), g[f"{tag}_{f}"]
            assert np.array_equal(a, b), f"{name} {tag} {f}: max diff {np.abs(a.astype(float) - b).max()}"

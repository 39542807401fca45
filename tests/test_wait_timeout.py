"""The bounded bulk-copy waits of the TMA cell kernel report a timeout
instead of hanging.

``tlm_gpu_set_test_wait_pad`` makes every wait of a mesh's TMA cell kernel
expect 16 bytes more than its copies bring.  The copies complete, the waits
cannot, so each runs out after its 2 s limit; the kernel records the error
word and returns, ``tlm_gpu_synchronize`` reports TLM_E_TIMEOUT, and a fresh
mesh on the same device afterwards runs and matches the oracle.  The CPU
test checks the hook's argument checks."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import build_tables, probe_series

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle  # noqa: E402


def small():
    return build_tables(cases.pml_point_source(24, pml=4, steps=20, dl=0.01, n_probes=2))


@pytest.mark.gpu
def test_gpu_bulk_wait_runs_out_and_reports(gpu_lib):
    t = small()
    g = capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32)
    g.set_variant(1)  # a TMA variant
    capi._check(capi._lib.tlm_gpu_set_test_wait_pad(g.h, 16))
    g.run(1, sync=False)
    with pytest.raises(capi.TLMError) as e:
        g.synchronize()
    assert e.value.code == capi.TLM_E_TIMEOUT
    g.close()
    # the device context is still usable
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as h:
        h.set_variant(1)
        h.run(int(t["n_timesteps"]))
        got = probe_series(t, h.cell_output())
    want = probe_series(t, oracle.Oracle(t).run(int(t["n_timesteps"])))
    assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want)


def test_wait_pad_arguments():
    """Argument checks only (a bad handle): no device call is made."""
    from ggi_tlm_b200 import build

    build.build()
    lib = capi.load_library()
    assert lib.tlm_gpu_set_test_wait_pad(123456789, 16) == capi.TLM_E_BADARG

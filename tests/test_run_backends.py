"""Backend selection of ksim_b200.run (CPU; no device work).

The reference's ``_run_sampler`` (src/python/ksim/run.py:79-91) accepts
"gpu", "cpu" and "auto" and raises ValueError for anything else.  This
package keeps "gpu" (as an alias of "b200") and "auto", and refuses "cpu"
loudly rather than falling back to a CPU path.
"""
from __future__ import annotations

import pytest


def test_unknown_and_cpu_backends_are_refused():
    from ksim_b200.run import resolve_backend
    with pytest.raises(ValueError, match="unknown backend"):
        resolve_backend("tpu")
    with pytest.raises(ValueError, match="sample_flat"):
        resolve_backend("cpu")
    assert resolve_backend("b200") == "b200"
    assert resolve_backend("gpu") == "b200"


def test_auto_needs_a_device():
    from ksim_b200 import _abi
    from ksim_b200.run import resolve_backend
    if _abi.lib().ksim_device_count() > 0:
        assert resolve_backend("auto") == "b200"
    else:
        with pytest.raises(RuntimeError, match="no CUDA device"):
            resolve_backend("auto")

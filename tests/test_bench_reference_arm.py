"""bench.py's reference arm on the CPU: the compiled reference (else the C
restatement) timed on its bounded sample, with the fields the JSON line
carries."""
import os

import pytest

from tests.conftest import REF_LIB


def test_cpu_reference_sample():
    import bench
    if not os.path.exists(REF_LIB) and not os.path.exists(bench.PORT_LIB):
        pytest.skip("no CPU build of the reference or the port")
    res, why = bench.cpu_reference(1, warmup=0)
    assert why is None
    assert res["value"] > 0 and res["cores"] == 1
    assert res["kind"] == ("reference" if os.path.exists(REF_LIB) else "port")
    assert "Q=" in res["sample"] and len(res["per_step_s"]) == 1

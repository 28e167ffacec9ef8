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


@pytest.mark.parametrize("kind", ["cfg2", "cfg3"])
def test_cpu_reference_batched_and_served_sample(kind):
    """The batched and served CPU baselines: the compiled reference on a
    sample of the systems, dealt to independent processes, rates summed."""
    import bench
    if not os.path.exists(REF_LIB):
        pytest.skip("needs the compiled reference")
    res, why = bench.cpu_reference_batch(kind, nsys=2, steps=1, procs=2)
    assert why is None
    assert res["value"] > 0 and res["cores"] == 2 and res["kind"] == "reference"
    if kind == "cfg3":
        assert res["latency_ms"]["p99"] >= res["latency_ms"]["p50"] > 0

"""CPU: the bench's workload constants and roofline arithmetic (bench.py), without running it."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_algorithmic_bytes_per_column_of_the_si216_block(bench):
    # 2 n_pw s + 2 N s + 8 N / nb, s = 16 B: 61,565 plane waves, 108^3 box, 452 columns
    assert bench.bytes_per_column(61565, 108 ** 3, 452) == pytest.approx(42_303_160, rel=1e-6)


def test_default_line_is_the_si216_block(bench, monkeypatch):
    monkeypatch.setattr("sys.argv", ["bench.py"])
    a = bench.parse()
    assert (a.gpus, a.impl, a.cell, a.workload) == (1, "ours", "si216", "hpsi")
    assert a.warmup >= 3 and not a.no_scf and not a.autotune
    w = bench.WORKLOADS[a.cell]
    assert (w["cell"], w["ecut"], w["kmesh"], w["nbands"]) == ("si216", 25.0, (1, 1, 1), 448)
    for key, path in bench.DRAM_SOURCE.items():  # the traffic figures cite committed summaries
        assert key in bench.LOCAL_DRAM_BYTES_PER_COLUMN
        assert os.path.exists(os.path.join(ROOT, path)), path

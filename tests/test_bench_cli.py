"""bench.py keeps its command-line contract (no GPU needed): every workload
the parser accepts has a runner, and the reference arm prints one JSON line."""
import importlib.util
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(HERE, "..", "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_every_workload_has_a_runner():
    b = _bench()
    assert callable(b.run_dense)
    assert callable(b.main)
    assert callable(b.run_reference_arm)
    assert callable(b.run_multimod)
    assert b.make_matrix(0.02).nr > 0
    assert b.multimod_matrix().nr == 500


def test_clock_summary_reports_median_and_throttle_reasons():
    b = _bench()
    clk = b.Clocks(0)
    clk.thread = object()  # the NVML sampler ran: summarise its samples
    clk.samples = [(1965, 1965, 0x0), (1950, 1965, 0x4), (1965, 1965, 0x4), (1800, 1965, 0x40)]
    out = clk.summary()
    assert out["sm_mhz"] == 1957.5 and out["sm_max_mhz"] == 1965
    assert out["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert out["samples"] == 4


def test_clock_summary_reads_nvidia_smi_csv(tmp_path):
    b = _bench()
    clk = b.Clocks(0)
    path = tmp_path / "clocks.csv"
    path.write_text("0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active\n"
                    "0, 1320, 1965, 1000.2, 0x4, Not Active, Not Active, Not Active, Active\n"
                    "0, 1400, 1965, 998.0, 0x4, Active, Not Active, Not Active, Active\n")
    clk.path = str(path)
    out = clk.summary()
    assert out["sm_mhz"] == 1400 and out["sm_max_mhz"] == 1965 and out["samples"] == 3
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"]


def test_reference_call_reduces_the_whole_matrix():
    """The CPU baseline is one call of the reference la on the whole matrix:
    its answer is the oracle's, and the baseline entry states the call's
    time and thread count without extrapolating."""
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    b = _bench()
    from gb_b200 import synth
    mat = synth.staircase(800, 200, 800, 65521, seed=3)
    ans, secs = b.reference_call(mat, 2)
    assert secs > 0 and ans.equals(oracle.oracle_la(mat)[0])
    cb = b.cpu_baseline_full(mat, 2, secs)
    assert cb["kind"] == "reference" and cb["cores"] == 2
    assert abs(cb["value"] - 1.0 / secs) < 1e-9 and "nothing extrapolated" in cb["sample"]


def test_both_arms_print_the_same_config():
    b = _bench()
    cfg = b.config_dict()
    assert cfg["workload"] == b.workload_name() and set(cfg) == {"workload", "l2"}


def test_multimod_cpu_baseline_scales_the_sampled_images():
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    b = _bench()
    cb = b.multimod_cpu_reference(b.multimod_matrix(), primes_used=100, lift_s=1.0, sample=2)
    assert cb["kind"] == "reference" and 0 < cb["value"] < 1.0
    assert "x 100 primes" in cb["sample"]

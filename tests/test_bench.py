"""The benchmark's bookkeeping without a GPU: the DRAM traffic the default line reports is the
ncu capture of the current kernel build, and the algorithmic bytes follow their formula."""

import bench


def test_the_default_workload_finds_its_traffic_capture():
    entry = bench.traffic_entry("fp64", "curves", bench.DEVICES_PER_GPU, bench.NP)
    assert entry is not None
    assert bench.KERNEL_TAG in entry["kernel"]
    assert entry["dram_bytes_per_launch"] == entry["read"] + entry["write"]
    assert bench.traffic_entry("fp64", "curves", bench.DEVICES_PER_GPU, 100) is None


def test_step_bytes_formula():
    # NP 400, FP64: NP [2 (9 + 3 (1 + K')) 8 + 48 + 8 n_stat] = 99.2 KB without ions,
    # 105.6 KB frozen (n_stat 3), 137.6 KB with the border (K' = 2)
    assert bench.step_bytes(400, False, False) == 99200
    assert bench.step_bytes(400, False, True) == 105600
    assert bench.step_bytes(400, True, False) == 137600
    assert bench.poisson_bytes(400) == 400 * 48

"""bench.py's tables agree with one another (CPU only): every roofline kernel has a byte model,
every recorded DRAM traffic names a known kernel and workload, and the default workloads exist
both in bench.py and in the library's workload table."""
import inspect
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import axoncuda_b200 as ax  # noqa: E402


def test_roofline_kernels_have_byte_models():
    for wl, kernel in bench.ROOFLINE_KERNELS.items():
        assert wl in bench.WORKLOADS, wl
        assert kernel in bench.BYTE_MODELS, kernel


def test_profiled_traffic_names_known_pairs():
    for (kernel, wl), traffic in bench.PROFILED_TRAFFIC.items():
        assert kernel in bench.BYTE_MODELS and wl in bench.WORKLOADS
        assert isinstance(traffic, int) and traffic > 0
    # the line's own pair has a capture
    line_kernel = bench.ROOFLINE_KERNELS[bench.DEFAULT_WORKLOAD]
    assert (line_kernel, bench.DEFAULT_WORKLOAD) in bench.PROFILED_TRAFFIC


def test_default_workloads_exist_in_both_tables():
    names = [bench.DEFAULT_WORKLOAD] + bench.DEFAULT_CONFIGS
    src = inspect.getsource(ax.workload)
    for name in names + ["snn-100k-incc"]:
        assert name in bench.WORKLOADS, name
        assert f'"{name}"' in src, name
    assert bench.DEFAULT_WORKLOAD not in bench.DEFAULT_CONFIGS


def test_sub_configs_default_to_one_gpu_runs():
    assert bench.sub_configs(None, 1) == bench.DEFAULT_CONFIGS
    assert bench.sub_configs(None, 8) == []
    assert bench.sub_configs("none", 1) == []
    assert bench.sub_configs("snn-8x512,circuit-200k-k64", 4) == ["snn-8x512", "circuit-200k-k64"]

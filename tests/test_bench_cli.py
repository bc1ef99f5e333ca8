"""The benchmark's command line on CPU: every mode it documents parses and has
its entry function (the GPU legs themselves run on the GPU machine)."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_modes_exist():
    sys.path.insert(0, ROOT)
    import bench
    for name in ('run_b200', 'run_reference', 'profile_case', 'cpu_baseline', 'fp64_comparison',
                 'whole_catalogue_comparison', 'reference_kernel_sample', 'distortion_sample', 'e2e_itemised',
                 'alu_roofline', 'smem_atomic_term', 'xi_errors'):
        assert callable(getattr(bench, name)), name


def test_bench_help_lists_the_modes():
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--help'], capture_output=True, text=True,
                         check=True).stdout
    for flag in ('--gpus', '--steps', '--warmup', '--impl', '--split', '--profile-case'):
        assert flag in out, flag

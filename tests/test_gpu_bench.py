"""bench.py on the device: one small run prints one JSON line with every key of
the benchmark contract (value, e2e with copy sizes, roofline with the measured
kernel time, clocks, launch count)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def test_bench_prints_the_contract_line():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    out = subprocess.run([sys.executable, str(ROOT / 'bench.py'), '--steps', '3', '--warmup', '3', '--structures', '16',
                          '--no-cpu-baseline', '--no-serve', '--no-autotune'],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better', 'scaling',
                'vs_baseline', 'dtype', 'data', 'config', 'e2e', 'roofline', 'clocks', 'gpu_launches'):
        assert key in d, key
    assert d['value'] > 0 and d['steps'] == 3 and d['warmup'] == 3 and d['n_gpus'] == 1
    assert d['e2e']['value'] > 0 and d['e2e']['h2d_bytes_per_step'] > 0 and d['e2e']['d2h_bytes_per_step'] > 0
    roof = d['roofline']
    assert roof['achieved'] > 0 and roof['peak'] > 0 and 0 < roof['frac'] < 1.5 and roof['kernel_ms'] > 0
    assert d['gpu_launches'] == 15 * 3
    assert d['ccs_rel_err_max_vs_fp64_oracle'] <= 1e-5
    # every timed block checked against the oracle on its own rays
    ccs = d['ccs_vs_fp64_oracle']
    assert ccs['blocks_checked'] == ccs['blocks'] == 16 * 3 and ccs['structure_rel_err_max'] <= 1e-5
    assert roof['ref_sphere_tests_per_ray'] > 0 and roof['ref_box_tests_per_ray'] > 0
    for name in ('C1_triatomic', 'C2_globule650', 'C3_globule2000'):
        c = d['configs'][name]
        assert c['rays_per_s'] > 0 and 0 < c['roofline_frac'] < 1.5 and c['ccs_rel_err_max_vs_fp64_oracle'] <= 1e-5
        assert sum(c['bounce_histogram']) == c['rays']
    assert d['configs']['C2_globule650']['pa_blocked_rays_equal_oracle'] is True
    assert d['e2e_explicit']['rays_per_s'] > 0
    assert d['plain']['rays_per_s'] > 0 and d['batched_over_plain'] > 0

"""ccs.py on the device against the reference CLI: the output files' layout
(tests/golden/cli_interface.json), the single-carbon example against its
analytic cross section, and four of the reference's own protein inputs
(tests/golden/structures.*: 1AL1, 1CLL, 1AO6 and 1BMF, 92 to 22,663 atoms)
read, prepared and traced exactly as the reference's solve_frame did
(16,384 rays x 3 replicates, seed 190003, EHSS and BVH PA, caps 64 and 512)."""
import hashlib
import json
import math
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / 'tests' / 'golden'


@pytest.fixture(scope='module')
def cli():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from ehss_b200 import ccs_cli
    return ccs_cli


def test_output_files_have_the_reference_layout(cli, tmp_path):
    ref = json.loads((GOLDEN / 'cli_interface.json').read_text(encoding='utf-8'))['results']
    xyz = ROOT / 'examples' / 'single_carbon.xyz'
    run = tmp_path / 'run'
    assert cli.main([str(xyz), '--rays', '1024', '--directions', '8', '--grid-size', '64', '--repeats', '2',
                     '--output', str(run)]) == 0
    payload = json.loads((run / 'results.json').read_text(encoding='utf-8'))
    rec = payload['records'][0]
    assert set(ref['top']) <= set(payload) and set(ref['record']) <= set(rec)
    assert set(ref['summary']) == set(rec['summary'])
    row = rec['runs'][0]
    assert set(ref['run']) == set(row) and set(ref['run_pa']) == set(row['pa'])
    assert set(ref['run_ehss']) <= set(row['ehss']) and set(ref['timings']) <= set(rec['timings'])
    assert set(payload['settings']) == set(ref['settings'])
    assert {k: v for k, v in payload['settings'].items() if k not in ('xyz', 'output')} == \
           {k: v for k, v in ref['settings'].items() if k not in ('xyz', 'output')}
    assert isinstance(row['ehss']['box_tests'], int) and row['ehss']['sphere_tests'] > 0
    header = (run / 'summary.csv').read_text(encoding='utf-8-sig').splitlines()[0].split(',')
    assert header == ref['csv_header']
    bvh = tmp_path / 'bvh'
    assert cli.main([str(xyz), '--rays', '1024', '--repeats', '1', '--pa-method', 'bvh', '--output', str(bvh)]) == 0
    row = json.loads((bvh / 'results.json').read_text(encoding='utf-8'))['records'][0]['runs'][0]
    assert set(row) == set(ref['run_bvh']) and set(row['pa']) == set(ref['run_pa_bvh'])
    # a lone sphere: a ray whose path crosses the sphere's box tests the sphere once (PA), or once
    # per query that does not start on it (EHSS); EHSS and PA trace the same 1024 rays
    assert 1000 <= row['pa']['sphere_tests'] <= 1024 and 1000 <= row['ehss']['sphere_tests'] <= 1024


def test_single_carbon_example_is_pi_r_squared(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    out = subprocess.run([sys.executable, str(ROOT / 'ccs.py'), str(ROOT / 'examples' / 'single_carbon.xyz'),
                          '--method', 'both', '--pa-method', 'bvh', '--rays', '16384', '--output',
                          str(tmp_path / 'run')], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    rec = json.loads((tmp_path / 'run' / 'results.json').read_text())['records'][0]
    exact = math.pi * 3.1 ** 2          # C: 1.70 A + 1.4 A probe; 30.1907 A^2
    for key in ('ehss_angstrom2', 'pa_angstrom2'):
        assert abs(rec['summary'][key]['mean'] - exact) <= 1e-6 * exact, key


STRUCTURES = json.loads((GOLDEN / 'structures.json').read_text())


@pytest.mark.parametrize('name', sorted(STRUCTURES))
def test_reference_structures_match_the_reference_cli(cli, tmp_path, name):
    """Read and prepared as the reference does (sphere arrays hash equal),
    then traced twice on the device: (a) the reference's own rays (the oracle's
    restatement of its numpy source, bit-exact to it) through the explicit-ray
    engine, which must give the reference's CCS, histograms and unresolved
    counts; (b) the CLI's fused path on its device-made rays, which must equal
    the oracle on those same rays.  The two ray sets agree to the last ulp or
    so (CUDA's and numpy's cosine and sine); multi-bounce paths through a large
    protein amplify that, so (a) and (b) are compared with the reference each
    on identical rays, and with one another only to the sampling level."""
    import ehss_b200 as eb
    from oracle import oracle as O
    entry = STRUCTURES[name]
    text = np.load(GOLDEN / 'structures.npz')[name].tobytes()
    xyz = tmp_path / f'{name}.xyz'
    xyz.write_bytes(text)
    frame = cli.read_xyz(xyz)[0]
    spheres, info = cli.prepare_frame(frame, cli.radius_table(None), 1.4)
    c, r = spheres.centers, spheres.radii
    assert len(r) == entry['atoms'] and info['comment'] == entry['comment']
    assert hashlib.sha256(np.ascontiguousarray(c).tobytes()).hexdigest() == entry['centers_sha256']
    assert hashlib.sha256(np.ascontiguousarray(r).tobytes()).hexdigest() == entry['radii_sha256']
    prep = eb.PreparedStaticGPUEHSS(spheres, precision='fp32')
    tree = O.StaticTree(c, r, 4)
    for cap, run in entry['runs'].items():
        cap = int(cap)
        # (a) the reference's rays on the device
        for ref_row in run['runs']:
            src = O.external_source(c, r, 14, ref_row['seed'])
            got = prep.engine.trace(eb.EHSSSource(src['origins'], src['directions'], src['incoming'], src['weights'],
                                                  src['last_atom'], src['initial_bounces'], 'reference rays'), cap)
            counts = np.bincount(got.bounces, minlength=cap + 1).tolist()
            assert counts == ref_row['ehss']['collision_histogram'], (name, cap, ref_row['seed'])
            assert int(got.unresolved.sum()) == ref_row['ehss']['unresolved_rays']
            assert got.omega == pytest.approx(ref_row['ehss']['ehss_angstrom2'], rel=1e-13)
            assert got.tail_bound == pytest.approx(ref_row['ehss']['tail_bound_angstrom2'], rel=1e-13, abs=1e-13)
            assert got.pa == pytest.approx(ref_row['ehss']['pa_from_same_rays_angstrom2'], rel=1e-13)
        # (b) the CLI's fused path equals the oracle on its own device rays
        argv = [a for a in run['argv'] if a != 'unused.xyz']
        argv[argv.index('--output') + 1] = str(tmp_path / f'out{cap}')
        out = cli.solve_frame(spheres, cli.parser().parse_args(['x.xyz'] + argv), progress=False)
        for row in out['runs']:
            o, d = (x.cpu().numpy() for x in prep.scene.source_rays(14, row['seed']))
            res = tree.trace(o, d, cap=cap, threads=O.host_cores())
            ro = O.readout(dict(incoming=d, weights=np.full(len(o), np.pi * prep.scene.radius ** 2 / len(o))), res, cap)
            assert row['ehss']['ehss_angstrom2'] == pytest.approx(ro['ehss_angstrom2'], rel=1e-12)
            assert row['ehss']['collision_histogram'] == ro['collision_histogram']
            hits, _, _ = O.PATree(c, r, 4).query(o, d, threads=O.host_cores())
            assert row['pa']['pa_angstrom2'] == pytest.approx(float(hits.sum()) * np.pi * prep.scene.radius ** 2 / len(o),
                                                             rel=1e-12)
        # the two ray sets sample the same cross section
        ref_mean = run['summary']['ehss_angstrom2']['mean']
        assert abs(out['summary']['ehss_angstrom2']['mean'] - ref_mean) <= 0.01 * ref_mean

"""The ccs.py interface against the reference CLI's own behaviour
(tests/golden/cli_interface.json, written by make_golden.py from the
reference): validation messages, the XYZ dialect and its error messages, the
radii JSON rules, frame preparation (bit-identical spheres), the defaults and
the summary.csv columns.  Host logic only: no device needed."""
import json
from pathlib import Path

import numpy as np
import pytest

from ehss_b200 import ccs_cli

GOLDEN = Path(__file__).resolve().parent / 'golden'


@pytest.fixture(scope='module')
def ref():
    return json.loads((GOLDEN / 'cli_interface.json').read_text(encoding='utf-8'))


def _parse(argv, output='/nonexistent/out'):
    return ccs_cli.parser().parse_args(['x.xyz', '--output', output, *argv])


def test_validation_messages(ref, tmp_path):
    for argv, message in ref['args'].items():
        if argv == '<existing output>':
            args = _parse([], str(tmp_path))
            expected = message.replace('{output}', str(tmp_path))
        else:
            args = _parse(argv.split())
            expected = message
        if expected is None:
            ccs_cli.validate_args(args)
            continue
        with pytest.raises(ValueError) as e:
            ccs_cli.validate_args(args)
        assert str(e.value) == expected, argv


def test_xyz_errors_and_accepted_dialect(ref, tmp_path):
    BAD_XYZ, GOOD_XYZ = ref['inputs']['xyz'], ref['inputs']['xyz_ok']
    for name, message in ref['xyz'].items():
        f = tmp_path / f'{name}.xyz'
        f.write_text(BAD_XYZ[name], encoding='utf-8')
        with pytest.raises(ValueError) as e:
            ccs_cli.read_xyz(f)
        assert str(e.value) == message.replace('{path}', str(f)), name
    for name, frames in ref['xyz_ok'].items():
        f = tmp_path / f'{name}.xyz'
        f.write_text(GOOD_XYZ[name], encoding='utf-8')
        got = ccs_cli.read_xyz(f)
        assert len(got) == len(frames)
        for g, r in zip(got, frames):
            assert g.number == r['number'] and g.comment == r['comment'] and list(g.elements) == r['elements']
            np.testing.assert_array_equal(g.coordinates, np.array(r['coordinates']))


def test_radii_json_rules(ref, tmp_path):
    BAD_RADII = ref['inputs']['radii']
    for name, message in ref['radii'].items():
        f = tmp_path / f'{name}.json'
        f.write_text(json.dumps(BAD_RADII[name]), encoding='utf-8')
        with pytest.raises(ValueError) as e:
            ccs_cli.radius_table(f)
        assert str(e.value) == message, name
    f = tmp_path / 'ok.json'
    f.write_text(json.dumps({'xe': 2.16, 'C': 1.8}), encoding='utf-8')
    table = ccs_cli.radius_table(f)
    assert table['Xe'] == 2.16 and table['C'] == 1.8 and table['N'] == ccs_cli.VDW_RADII['N']
    assert ccs_cli.radius_table(None) == ref['results']['radii']


def test_frame_preparation_bit_identical(ref):
    table = ccs_cli.radius_table(None)
    frame = ccs_cli.XYZFrame
    cases = {
        'only_h_excluded': (frame(1, 'h', ('H', 'H'), np.array([[0., 0, 0], [1, 0, 0]])), dict(exclude_hydrogen=True)),
        'unknown': (frame(2, 'u', ('C', 'Xe', 'Au'), np.array([[0., 0, 0], [1, 0, 0], [2, 0, 0]])), {}),
        'coincident': (frame(3, 'c', ('C', 'O'), np.array([[1., 2, 3], [1, 2, 3]])), {}),
        'overflow': (frame(1, 'o', ('C', 'O'), np.array([[0., 0, 0], [1e308, 0, 0]])), dict(units='nm')),
        'ok_nm': (frame(4, 'ok', ('O', 'H', 'H'), np.array([[0.1, 0, 0], [0.2, 0.05, 0], [0, 0.3, 0.01]])),
                  dict(units='nm')),
        'ok_noh': (frame(5, 'ok', ('O', 'H', 'C'), np.array([[3., 1, 0], [2, 0.5, 0], [0, 3, 0.1]])),
                   dict(exclude_hydrogen=True)),
    }
    for name, (fr, kw) in cases.items():
        expected = ref['frames'][name]
        if isinstance(expected, str):
            with pytest.raises(ValueError) as e:
                ccs_cli.prepare_frame(fr, table, 1.4, **kw)
            assert str(e.value) == expected, name
        else:
            spheres, info = ccs_cli.prepare_frame(fr, table, 1.4, **kw)
            np.testing.assert_array_equal(spheres.centers, np.array(expected['centers']))
            np.testing.assert_array_equal(spheres.radii, np.array(expected['radii']))
            assert json.loads(json.dumps(info)) == expected['info'], name


def test_defaults_and_output_columns(ref):
    ours = {k: (str(v) if isinstance(v, Path) else v) for k, v in vars(ccs_cli.parser().parse_args(['x.xyz'])).items()}
    assert ours == ref['default_settings']
    assert [name for name, _ in ccs_cli.SUMMARY_COLUMNS] == ref['results']['csv_header']
    assert ccs_cli.RADII_SOURCE == ref['results']['radii_source']


def test_summary_csv_writer(tmp_path, ref):
    import csv
    rec = dict(input_file='a.xyz', frame=2, selected_atoms=7, timings=dict(all_replicates_with_setup_s=0.5),
               summary=dict(ehss_angstrom2=dict(mean=10.0, sd=None), ehss_tail_bound_mean_angstrom2=0.0,
                            ehss_unresolved_rays_total=0))
    ccs_cli.write_summary_csv(tmp_path / 's.csv', [rec])
    with (tmp_path / 's.csv').open(encoding='utf-8-sig', newline='') as f:
        rows = list(csv.DictReader(f))
    assert list(rows[0]) == ref['results']['csv_header']
    assert rows[0]['ehss_mean_A2'] == '10.0' and rows[0]['pa_mean_A2'] == '' and rows[0]['atoms'] == '7'


def test_main_exit_code_on_invalid_input(tmp_path):
    bad = tmp_path / 'bad.xyz'
    bad.write_text('2\ncomment\nC 0 0 0\n', encoding='utf-8')
    with pytest.raises(SystemExit) as e:
        ccs_cli.main([str(bad), '--output', str(tmp_path / 'out')])
    assert e.value.code == 2
    with pytest.raises(SystemExit) as e:
        ccs_cli.main([str(tmp_path / 'missing*.xyz'), '--output', str(tmp_path / 'out')])
    assert e.value.code == 2

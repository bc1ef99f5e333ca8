"""The multi-file drivers' host side, without a GPU: an empty data directory
ends the run with the reference's NameError ('Empty data. Did you write
correctly the input directory?', ``2pla_multiple_data.py`` /
``distortion_multiple_data.py``) before any device work."""
import os
import subprocess
import sys

import pytest

from lya2pcf_b200.dropin_path import DROPIN_DIR


@pytest.mark.parametrize('script, extra', [('2pla_multiple_data.py', ['--gpu']),
                                           ('distortion_multiple_data.py', ['--excluded', '0'])])
def test_empty_data_directory_raises(tmp_path, script, extra):
    ddir = tmp_path / 'deltas'
    ddir.mkdir()
    env = {k: v for k, v in os.environ.items() if k not in ('RANK', 'WORLD_SIZE', 'LOCAL_RANK')}
    r = subprocess.run([sys.executable, os.path.join(DROPIN_DIR, script), '--data-dir', str(ddir),
                        '--corr-dir', str(tmp_path / 'out')] + extra,
                       capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode != 0
    assert 'NameError: Empty data' in r.stderr

"""Persistence of the autotuners' choices (gpw_tune_export / gpw_tune_import).

A tuned launch leaves a record; exporting, saving, loading and importing the
records round-trips them; a file written for another device or SM count is
refused; a record naming a layout the shape does not have is skipped.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_export_import_round_trip(cuda, tmp_path):
    import torch
    from gpawdft_b200 import _lib, tuning
    from gpawdft_b200.fd_operators import Laplace
    from gpawdft_b200.grid_descriptor import GridDescriptor
    # a zero-boundary float64 apply (16-byte rows: the TMA kernel) and a
    # complex Bloch apply get tuned
    gd = GridDescriptor((41, 37, 45), (8.2, 7.4, 9.0), 0)
    a = torch.randn((3,) + tuple(gd.n_c), dtype=torch.float64, device='cuda')
    Laplace(gd, -0.5, 3).apply(a, torch.empty_like(a))
    gdp = GridDescriptor((32, 32, 64), (6.0, 6.0, 12.0), 1)
    b = torch.randn((2,) + tuple(gdp.n_c), dtype=torch.complex128,
                    device='cuda')
    ph = np.exp(2j * np.pi * gdp.sdisp_cd * 0.1)
    Laplace(gdp, -0.5, 3, complex).apply(b, torch.empty_like(b), ph)
    text = tuning.export_records()
    lines = text.strip().split('\n')
    assert lines[0].startswith('gpwgrid-tune 1 sms ')
    assert any(l.startswith('tma ') for l in lines)
    assert any(l.startswith('bloch ') for l in lines)
    path = os.path.join(str(tmp_path), 'tune.json')
    tuning.save(path)
    n = tuning.load(path)
    assert n == len(lines) - 1
    # another device's header is refused
    other = text.replace(' sms ', ' sms 1', 1)
    with pytest.raises(_lib.GPWError):
        tuning.import_records(other)
    # a record with a variant that does not exist is skipped
    bad = lines[0] + '\ntma 0 3 0 10 10 10 1 99 0\n'
    assert tuning.import_records(bad) == 0

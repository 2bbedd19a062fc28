import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "mmff_small.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


def batch_from_golden(d, tag):
    from firecore_b200.systems import SystemBatch
    keys = ['natoms', 'nnode', 'pos', 'neighs', 'neighCell', 'bkneighs', 'REQs', 'apars', 'bLs', 'bKs', 'Ksp', 'Kpp',
            'lvec', 'elements']
    return SystemBatch(*[d[f'{tag}_{k}'] for k in keys])


def grid_from_golden(d):
    from firecore_b200.systems import GridSpec
    return GridSpec(tuple(int(x) for x in d['grid_n']), tuple(float(x) for x in d['grid_pos0']),
                    tuple(float(x) for x in d['grid_step']))

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def inputs(tmp_path_factory):
    """Synthetic input files (.tri, .nmat) for the slab and grating workloads."""
    from nebula_b200.synth import workloads, geometry, materials, nmat
    d = tmp_path_factory.mktemp("inputs")
    out = {}
    slab = workloads.slab()
    geometry.write_tri(str(d / "slab.tri"), slab.triangles)
    gr = workloads.grating_geometry()
    geometry.write_tri(str(d / "grating.tri"), gr)
    nmat.write(str(d / "si.nmat"), materials.build_raw_material(materials.silicon()))
    nmat.write(str(d / "pmma.nmat"), materials.build_raw_material(materials.pmma()))
    nmat.write(str(d / "si_kieft.nmat"), materials.build_raw_material(materials.silicon(), inelastic="kieft"))
    nmat.write(str(d / "pmma_kieft.nmat"), materials.build_raw_material(materials.pmma(), inelastic="kieft"))
    out["dir"] = str(d)
    for k in ("slab.tri", "grating.tri", "si.nmat", "pmma.nmat", "si_kieft.nmat", "pmma_kieft.nmat"):
        out[k] = str(d / k)
    return out


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)

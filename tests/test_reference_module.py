"""FireCore's own, unmodified pyBall/MMFF_multi.py binds this library.

The reference module loads ``libMMFFmulti_lib.so`` from
``<pyBall>/../../cpp/Build/libs_OCL`` (pyBall/MMFF_multi.py:77-78,
pyBall/cpp_utils_.py:61-69) and declares the argtypes of all 43 functions at
import time.  The test copies the reference's pyBall package (read from the
FireCore tree where it lies; skipped where that tree is absent) into a
temporary tree, puts a link to this repository's library where the loader
looks, imports the module in a fresh process and calls the CPU-side
samplers through the reference's own Python wrappers, checking them against
closed-form values.  The GPU paths (init / run / eval) need a device and are
covered through this package's mirror of the module (test_gpu_legacy.py).
"""
import os
import shutil
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_ROOT = os.environ.get("REF_ROOT", "/root/reference")
PYBALL = os.path.join(REF_ROOT, "pyBall")
LIB = os.path.join(ROOT, "firecore_b200", "libMMFFmulti_lib.so")


@pytest.mark.skipif(not os.path.isfile(os.path.join(PYBALL, "MMFF_multi.py")), reason="FireCore tree not present")
def test_unmodified_pyball_module_binds_this_library(tmp_path):
    shutil.copytree(PYBALL, tmp_path / "pyBall", ignore=shutil.ignore_patterns("tests", "doc", "*.pyc"))
    libdir = tmp_path / "cpp" / "Build" / "libs_OCL"
    libdir.mkdir(parents=True)
    os.symlink(LIB, libdir / "libMMFFmulti_lib.so")
    code = textwrap.dedent(f"""
        import sys, numpy as np
        sys.path.insert(0, {str(tmp_path)!r})
        import pyBall.MMFF_multi as mmff
        assert hasattr(mmff.lib, "mmff_last_error"), "the reference module did not load this library"
        # pyBall/MMFF_multi.py:131-136 sample_evalAngleCosHalf (Forces.h:190)
        ang = np.linspace(0.5, 3.0, 7)
        E, F = mmff.sample_evalAngleCosHalf(ang, K=2.0, ang0=1.9)
        # E = K (1 - cos((a - a0) / 2)) of the cos-half form (MMFFsp3_loc apars convention)
        ref = 2.0 * (1.0 - np.cos((ang - 1.9) / 2))
        assert np.abs(E - ref).max() < 1e-9, (E, ref)
        # pyBall/MMFF_multi.py:101-106 sample_DistConstr, a flat-bottom spring
        xs = np.linspace(0.0, 3.0, 13)
        E2, F2 = mmff.sample_DistConstr(xs, lmin=1.0, lmax=2.0, kmin=1.5, kmax=0.5, flim=1e300)
        assert np.isfinite(E2).all() and (E2[(xs > 1.0) & (xs < 2.0)] == 0).all()
        print("ok", len([k for k in dir(mmff) if not k.startswith("_")]))
    """)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert "ok" in out.stdout

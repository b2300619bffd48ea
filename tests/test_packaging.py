"""The package installs and imports as ``mbd_icenav_b200`` (the source
directory's name has a hyphen; pyproject.toml maps it), with its built
library inside, and loads without the in-repo import helper."""
import glob
import os
import shutil
import subprocess
import sys

import pytest

from conftest import ROOT


def test_wheel_installs_and_imports(tmp_path):
    from mbd_icenav_b200 import build
    build.build_library()
    # build from a copy, so that setuptools' build folders stay out of the repository
    src = tmp_path / "src"
    shutil.copytree(os.path.join(ROOT, "mbd-icenav_b200"), src / "mbd-icenav_b200",
                    ignore=shutil.ignore_patterns("__pycache__"))
    shutil.copy(os.path.join(ROOT, "pyproject.toml"), src / "pyproject.toml")
    wheel_dir, target = tmp_path / "wheel", tmp_path / "site"
    r = subprocess.run([sys.executable, "-m", "pip", "wheel", "--no-deps", "--no-build-isolation", "--no-index",
                        "-w", str(wheel_dir), str(src)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    whl = glob.glob(str(wheel_dir / "*.whl"))
    assert len(whl) == 1
    r = subprocess.run([sys.executable, "-m", "pip", "install", "--no-deps", "--no-index", "--target", str(target),
                        whl[0]], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    code = ("import mbd_icenav_b200, os; from mbd_icenav_b200 import _abi, sim, planner; "
            "lib = _abi.load_library(); print(lib.dem_version().decode()); "
            "assert os.path.dirname(_abi.LIB_PATH) == os.path.dirname(mbd_icenav_b200.__file__)")
    env = dict(os.environ, PYTHONPATH=str(target))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env,
                       cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "sm_100a" in r.stdout

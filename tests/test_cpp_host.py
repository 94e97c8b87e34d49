"""The C++ host mirror (bismit_b200/cpp/bismit.hpp): its builders resolve
the same descriptors as the Python mirror, its errors carry the C status
codes, and a cortex built and cycled through Cortex::builder matches the
oracle. The test program is compiled with the system C++ compiler."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from bismit_b200 import _ffi as F, configs, map as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SIDES = (32, 48, 24)


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("cpp") / "test_cortex")
    libdir = os.path.join(ROOT, "bismit_b200")
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "bismit_b200", "cpp"),
           os.path.join(ROOT, "tests", "cpp", "test_cortex.cpp"), "-L", libdir, "-lbismit_b200",
           "-Wl,-rpath," + libdir, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def _py_desc(builder, name="v1"):
    lmaps, areas = builder()[:2]
    return bytes(M.area_desc(name, lmaps, areas, configs.bench_settings()))


def test_cpp_builders_resolve_the_python_descriptors(exe, tmp_path):
    r = subprocess.run([exe, "desc", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "errors ok" in r.stdout
    assert open(tmp_path / "area_64_v1.bin", "rb").read() == _py_desc(lambda: configs.workload("area_64"))
    assert open(tmp_path / "mixed_v1.bin", "rb").read() == _py_desc(lambda: configs.mixed_area(32, 48))
    from test_hierarchy import _with_filters
    for n in ("v1", "v2"):
        want = _py_desc(lambda: _with_filters(*configs.hierarchy(SIDES)[:2]), n)
        assert open(tmp_path / ("filtered_%s.bin" % n), "rb").read() == want, n
    lmaps, areas, names = configs.hierarchy(SIDES)
    for n in names:
        assert open(tmp_path / ("hierarchy_%s.bin" % n), "rb").read() == bytes(
            M.area_desc(n, lmaps, areas, configs.bench_settings())), n


@pytest.mark.gpu
def test_cpp_cortex_matches_oracle(exe, tmp_path):
    from helpers import oracle_cortex_cycle
    lmaps, areas, names = configs.hierarchy(SIDES)
    n = 5
    frames = configs.frames(n, SIDES[0] ** 2, 0.02, 8)
    frames.tofile(str(tmp_path / "frames.bin"))
    r = subprocess.run([exe, "cycle", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    plans = []
    for k, name in enumerate(names):
        d = M.area_desc(name, lmaps, areas, configs.bench_settings())
        p = F.bm_area_plan()
        F.check(F.lib().bm_plan_resolve(C.byref(d), 3, C.byref(p)))
        plans.append(p)
    slabs = [np.fromfile(str(tmp_path / ("init_%s.bin" % nm)), np.uint8) for nm in names]
    for k, (p, s) in enumerate(zip(plans, slabs)):
        ref = np.zeros(int(p.slab_bytes), np.uint8)
        oracle.grow(p, ref, 3, configs.bench_settings().init_flags)
        assert np.array_equal(ref, s), "growth of %s" % names[k]
    tracts, _ext = M.area_tracts(lmaps, areas, names, plans)
    for c in range(n):
        oracle_cortex_cycle(plans, slabs, tracts, frames[c], c)
    for k, nm in enumerate(names):
        dev = np.fromfile(str(tmp_path / ("final_%s.bin" % nm)), np.uint8)
        assert np.array_equal(dev, slabs[k]), nm
